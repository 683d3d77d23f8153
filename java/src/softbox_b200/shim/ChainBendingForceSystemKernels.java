package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of ChainBendingForceSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class ChainBendingForceSystemKernels {
    private ChainBendingForceSystemKernels() {}

    private static final MethodHandle H_ZERO_ACCUMULATORS = Sbx.h("sbx_zero_accumulators",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS));

    /** ChainBendingForceSystem.zeroAccumulators (ChainBendingForceSystem.java:38-45) -> sbx_zero_accumulators. */
    public static void zeroAccumulators(FloatArray forceSum, FloatArray torqueSum, IntArray counts) {
        Sbx.toDevice(forceSum, torqueSum);
        try {
            Sbx.check((int) H_ZERO_ACCUMULATORS.invokeExact(Sbx.ctx(), forceSum.getSize() / 3, forceSum.dev(), torqueSum.dev()), "sbx_zero_accumulators");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(forceSum, torqueSum);
    }

    private static final MethodHandle H_CHAIN_FORCES = Sbx.h("sbx_chain_forces",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** ChainBendingForceSystem.chainForces (ChainBendingForceSystem.java:105-331) -> sbx_chain_forces. */
    public static void chainForces(FloatArray coord, FloatArray uVec, FloatArray segLength, IntArray end2NbrSlot, IntArray end2NbrSide, IntArray end1NbrSlot, IntArray end1NbrSide, FloatArray bTransGam, FloatArray bRotGam, FloatArray forceSum, FloatArray torqueSum, FloatArray chainParams, IntArray counts) {
        Sbx.toDevice(coord, uVec, segLength, end2NbrSlot, end2NbrSide, end1NbrSlot, end1NbrSide, bTransGam, bRotGam, forceSum, torqueSum, chainParams);
        try {
            Sbx.check((int) H_CHAIN_FORCES.invokeExact(Sbx.ctx(), coord.getSize() / 3, coord.dev(), uVec.dev(), segLength.dev(), end2NbrSlot.dev(), end2NbrSide.dev(), end1NbrSlot.dev(), end1NbrSide.dev(), bTransGam.dev(), bRotGam.dev(), forceSum.dev(), torqueSum.dev(), chainParams.dev()), "sbx_chain_forces");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(forceSum, torqueSum);
    }

}
