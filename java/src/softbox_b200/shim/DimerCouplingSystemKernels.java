package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of DimerCouplingSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class DimerCouplingSystemKernels {
    private DimerCouplingSystemKernels() {}

    private static final MethodHandle H_DIMER_COUPLE = Sbx.h("sbx_dimer_couple",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** DimerCouplingSystem.couple (DimerCouplingSystem.java:83-184) -> sbx_dimer_couple. */
    public static void couple(FloatArray coord, FloatArray uVec, FloatArray segLength, FloatArray bTransGam, FloatArray bRotGam, FloatArray forceSum, FloatArray torqueSum, IntArray motorA, IntArray motorB, IntArray parallel, FloatArray dimerParams, IntArray boundSeg) {
        Sbx.toDevice(coord, uVec, segLength, bTransGam, bRotGam, forceSum, torqueSum, motorA, motorB, parallel, dimerParams, boundSeg);
        try {
            Sbx.check((int) H_DIMER_COUPLE.invokeExact(Sbx.ctx(), coord.getSize() / 3, coord.dev(), uVec.dev(), segLength.dev(), bTransGam.dev(), bRotGam.dev(), forceSum.dev(), torqueSum.dev(), motorA.getSize(), motorA.dev(), motorB.dev(), parallel.dev(), dimerParams.dev(), boundSeg.dev()), "sbx_dimer_couple");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(forceSum, torqueSum);
    }

}
