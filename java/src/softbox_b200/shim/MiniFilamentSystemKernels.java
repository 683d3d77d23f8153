package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of MiniFilamentSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class MiniFilamentSystemKernels {
    private MiniFilamentSystemKernels() {}

    private static final MethodHandle H_MINI_TETHER = Sbx.h("sbx_mini_tether",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** MiniFilamentSystem.tether (MiniFilamentSystem.java:65-134) -> sbx_mini_tether. */
    public static void tether(FloatArray mCoord, FloatArray mUVec, FloatArray mSegLength, FloatArray mBTransGam, FloatArray mBRotGam, FloatArray mForceSum, FloatArray mTorqueSum, FloatArray bbCoord, FloatArray bbUVec, FloatArray bbInvDragY, IntArray headBackboneSlot, IntArray motorA, FloatArray attachAxial, FloatArray miniData, FloatArray miniParams) {
        Sbx.toDevice(mCoord, mUVec, mSegLength, mBTransGam, mBRotGam, mForceSum, mTorqueSum, bbCoord, bbUVec, bbInvDragY, headBackboneSlot, motorA, attachAxial, miniData, miniParams);
        try {
            Sbx.check((int) H_MINI_TETHER.invokeExact(Sbx.ctx(), mCoord.getSize() / 3, mCoord.dev(), mUVec.dev(), mSegLength.dev(), mBTransGam.dev(), mBRotGam.dev(), mForceSum.dev(), mTorqueSum.dev(), bbCoord.getSize() / 3, bbCoord.dev(), bbUVec.dev(), bbInvDragY.dev(), headBackboneSlot.getSize(), headBackboneSlot.dev(), motorA.dev(), attachAxial.dev(), miniData.dev(), miniParams.dev()), "sbx_mini_tether");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(mForceSum, mTorqueSum, miniData);
    }

    private static final MethodHandle H_MINI_BACKBONE_GATHER = Sbx.h("sbx_mini_backbone_gather",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** MiniFilamentSystem.backboneGather (MiniFilamentSystem.java:137-155) -> sbx_mini_backbone_gather. */
    public static void backboneGather(IntArray bbDimerOffsets, IntArray bbDimerList, FloatArray miniData, FloatArray bbForceSum, FloatArray bbTorqueSum, IntArray miniCounts) {
        Sbx.toDevice(bbDimerOffsets, bbDimerList, miniData, bbForceSum, bbTorqueSum);
        try {
            Sbx.check((int) H_MINI_BACKBONE_GATHER.invokeExact(Sbx.ctx(), miniCounts.get(3), bbDimerOffsets.dev(), bbDimerList.dev(), miniData.dev(), bbForceSum.dev(), bbTorqueSum.dev()), "sbx_mini_backbone_gather");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(bbForceSum, bbTorqueSum);
    }

}
