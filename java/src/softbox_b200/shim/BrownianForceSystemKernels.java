package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of BrownianForceSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class BrownianForceSystemKernels {
    private BrownianForceSystemKernels() {}

    private static final MethodHandle H_BROWNIAN_FORCE = Sbx.h("sbx_brownian_force",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** BrownianForceSystem.brownianForce (BrownianForceSystem.java:44-106) -> sbx_brownian_force. */
    public static void brownianForce(FloatArray randForce, FloatArray randTorque, FloatArray bTransGam, FloatArray bRotGam, FloatArray brownTransScale, FloatArray brownRotScale, FloatArray params, IntArray counts) {
        Sbx.toDevice(randForce, randTorque, bTransGam, bRotGam, brownTransScale, brownRotScale, params, counts);
        try {
            Sbx.check((int) H_BROWNIAN_FORCE.invokeExact(Sbx.ctx(), randForce.getSize() / 3, randForce.dev(), randTorque.dev(), bTransGam.dev(), bRotGam.dev(), brownTransScale.dev(), brownRotScale.dev(), params.dev(), counts.dev()), "sbx_brownian_force");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(randForce, randTorque);
    }

}
