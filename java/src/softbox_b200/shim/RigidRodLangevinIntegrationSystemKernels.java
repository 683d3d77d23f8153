package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of RigidRodLangevinIntegrationSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class RigidRodLangevinIntegrationSystemKernels {
    private RigidRodLangevinIntegrationSystemKernels() {}

    private static final MethodHandle H_INTEGRATE = Sbx.h("sbx_integrate",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** RigidRodLangevinIntegrationSystem.integrate (RigidRodLangevinIntegrationSystem.java:33-112) -> sbx_integrate. */
    public static void integrate(FloatArray coord, FloatArray uVec, FloatArray yVec, FloatArray forceSum, FloatArray torqueSum, FloatArray randForce, FloatArray randTorque, FloatArray bTransGam, FloatArray bRotGam, FloatArray params, IntArray counts) {
        Sbx.toDevice(coord, uVec, yVec, forceSum, torqueSum, randForce, randTorque, bTransGam, bRotGam, params);
        try {
            Sbx.check((int) H_INTEGRATE.invokeExact(Sbx.ctx(), coord.getSize() / 3, coord.dev(), MemorySegment.NULL, uVec.dev(), yVec.dev(), forceSum.dev(), torqueSum.dev(), randForce.dev(), randTorque.dev(), bTransGam.dev(), bRotGam.dev(), params.dev()), "sbx_integrate");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(coord, uVec, yVec);
    }

}
