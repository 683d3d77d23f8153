package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of CrosslinkerSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class CrosslinkerSystemKernels {
    private CrosslinkerSystemKernels() {}

    private static final MethodHandle H_XLINK_COUNT_ACTIVE = Sbx.h("sbx_xlink_count_active",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_INT, ADDRESS));

    /** CrosslinkerSystem.countActiveLinks (CrosslinkerSystem.java:694-706) -> sbx_xlink_count_active. */
    public static void countActiveLinks(IntArray linkState, IntArray linkFilA, IntArray linkFilB, IntArray activeLinkCount, IntArray formCounts) {
        Sbx.toDevice(linkState, linkFilA, linkFilB, activeLinkCount);
        try {
            Sbx.check((int) H_XLINK_COUNT_ACTIVE.invokeExact(Sbx.ctx(), linkState.getSize(), linkState.dev(), linkFilA.dev(), linkFilB.dev(), activeLinkCount.getSize(), activeLinkCount.dev()), "sbx_xlink_count_active");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(activeLinkCount);
    }

    private static final MethodHandle H_XLINK_FORCES = Sbx.h("sbx_xlink_forces",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** CrosslinkerSystem.linkForces (CrosslinkerSystem.java:51-124) -> sbx_xlink_forces. */
    public static void linkForces(FloatArray filCoord, FloatArray filUVec, FloatArray filEnd1, FloatArray filBTransGam, IntArray linkFilA, IntArray linkFilB, FloatArray loc1, FloatArray loc2, IntArray filLinkCt, FloatArray xlinkData, FloatArray xlParams) {
        Sbx.toDevice(filCoord, filUVec, filEnd1, filBTransGam, linkFilA, linkFilB, loc1, loc2, filLinkCt, xlinkData, xlParams);
        try {
            Sbx.check((int) H_XLINK_FORCES.invokeExact(Sbx.ctx(), filCoord.getSize() / 3, filCoord.dev(), filUVec.dev(), filEnd1.dev(), filBTransGam.dev(), linkFilA.getSize(), linkFilA.dev(), linkFilB.dev(), loc1.dev(), loc2.dev(), filLinkCt.dev(), xlinkData.dev(), xlParams.dev()), "sbx_xlink_forces");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(xlinkData);
    }

    private static final MethodHandle H_XLINK_TORSION = Sbx.h("sbx_xlink_torsion",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** CrosslinkerSystem.linkTorsion (CrosslinkerSystem.java:767-808) -> sbx_xlink_torsion. */
    public static void linkTorsion(FloatArray filUVec, IntArray linkFilA, IntArray linkFilB, IntArray linkState, IntArray linkOrientSame, FloatArray torqueMagHist, IntArray torqueMagPlace, FloatArray xlinkData, FloatArray torsionParams) {
        Sbx.toDevice(filUVec, linkFilA, linkFilB, linkState, linkOrientSame, torqueMagHist, torqueMagPlace, xlinkData, torsionParams);
        try {
            Sbx.check((int) H_XLINK_TORSION.invokeExact(Sbx.ctx(), filUVec.getSize() / 3, filUVec.dev(), linkFilA.getSize(), linkFilA.dev(), linkFilB.dev(), linkState.dev(), linkOrientSame.dev(), torqueMagHist.dev(), torqueMagPlace.dev(), xlinkData.dev(), torsionParams.dev()), "sbx_xlink_torsion");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(torqueMagHist, torqueMagPlace, xlinkData);
    }

    private static final MethodHandle H_XLINK_SEG_GATHER = Sbx.h("sbx_xlink_seg_gather",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** CrosslinkerSystem.segGatherA (CrosslinkerSystem.java:129-149) -> sbx_xlink_seg_gather. */
    public static void segGatherA(IntArray segOffsets, IntArray segLinkIdx, FloatArray xlinkData, IntArray linkState, FloatArray filForceSum, FloatArray filTorqueSum, IntArray counts) {
        Sbx.toDevice(segOffsets, segLinkIdx, xlinkData, linkState, filForceSum, filTorqueSum);
        try {
            Sbx.check((int) H_XLINK_SEG_GATHER.invokeExact(Sbx.ctx(), 0, counts.get(3), segOffsets.dev(), segLinkIdx.dev(), xlinkData.dev(), linkState.dev(), filForceSum.dev(), filTorqueSum.dev()), "sbx_xlink_seg_gather");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(filForceSum, filTorqueSum);
    }

    private static final MethodHandle H_XLINK_SEG_GATHER_1 = Sbx.h("sbx_xlink_seg_gather",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** CrosslinkerSystem.segGatherB (CrosslinkerSystem.java:153-173) -> sbx_xlink_seg_gather. */
    public static void segGatherB(IntArray segOffsets, IntArray segLinkIdx, FloatArray xlinkData, IntArray linkState, FloatArray filForceSum, FloatArray filTorqueSum, IntArray counts) {
        Sbx.toDevice(segOffsets, segLinkIdx, xlinkData, linkState, filForceSum, filTorqueSum);
        try {
            Sbx.check((int) H_XLINK_SEG_GATHER_1.invokeExact(Sbx.ctx(), 1, counts.get(3), segOffsets.dev(), segLinkIdx.dev(), xlinkData.dev(), linkState.dev(), filForceSum.dev(), filTorqueSum.dev()), "sbx_xlink_seg_gather");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(filForceSum, filTorqueSum);
    }

    private static final MethodHandle H_XLINK_UNBIND = Sbx.h("sbx_xlink_unbind",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** CrosslinkerSystem.unbind (CrosslinkerSystem.java:231-281) -> sbx_xlink_unbind. */
    public static void unbind(FloatArray filCoord, FloatArray filUVec, FloatArray filEnd1, IntArray linkFilA, IntArray linkFilB, FloatArray loc1, FloatArray loc2, IntArray linkState, FloatArray strainHist, IntArray strainPlace, FloatArray offParams, IntArray counts) {
        Sbx.toDevice(filUVec, filEnd1, linkFilA, linkFilB, loc1, loc2, linkState, strainHist, strainPlace, offParams, counts);
        try {
            Sbx.check((int) H_XLINK_UNBIND.invokeExact(Sbx.ctx(), filCoord.getSize() / 3, filUVec.dev(), filEnd1.dev(), counts.get(0), linkFilA.dev(), linkFilB.dev(), loc1.dev(), loc2.dev(), linkState.dev(), strainHist.dev(), strainPlace.dev(), offParams.dev(), counts.dev()), "sbx_xlink_unbind");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(linkState, strainHist, strainPlace);
    }

}
