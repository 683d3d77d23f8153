package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of DerivedGeometrySystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class DerivedGeometrySystemKernels {
    private DerivedGeometrySystemKernels() {}

    private static final MethodHandle H_DERIVE = Sbx.h("sbx_derive",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** DerivedGeometrySystem.derive (DerivedGeometrySystem.java:27-73) -> sbx_derive. */
    public static void derive(FloatArray coord, FloatArray uVec, FloatArray yVec, FloatArray zVec, FloatArray end1, FloatArray end2, FloatArray segLength, IntArray counts) {
        Sbx.toDevice(coord, uVec, yVec, zVec, end1, end2, segLength);
        try {
            Sbx.check((int) H_DERIVE.invokeExact(Sbx.ctx(), coord.getSize() / 3, coord.dev(), uVec.dev(), yVec.dev(), zVec.dev(), end1.dev(), end2.dev(), segLength.dev()), "sbx_derive");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(yVec, zVec, end1, end2);
    }

}
