package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of ContainmentSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class ContainmentSystemKernels {
    private ContainmentSystemKernels() {}

    private static final MethodHandle H_CONFINE = Sbx.h("sbx_confine",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** ContainmentSystem.confine (ContainmentSystem.java:58-126) -> sbx_confine. */
    public static void confine(FloatArray coord, FloatArray uVec, FloatArray segLength, FloatArray bTransGam, FloatArray forceSum, FloatArray torqueSum, FloatArray boxParams, IntArray counts) {
        Sbx.toDevice(coord, uVec, segLength, bTransGam, forceSum, torqueSum, boxParams, counts);
        try {
            Sbx.check((int) H_CONFINE.invokeExact(Sbx.ctx(), coord.getSize() / 3, coord.dev(), uVec.dev(), segLength.dev(), bTransGam.dev(), forceSum.dev(), torqueSum.dev(), boxParams.dev(), counts.dev()), "sbx_confine");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(forceSum, torqueSum);
    }

}
