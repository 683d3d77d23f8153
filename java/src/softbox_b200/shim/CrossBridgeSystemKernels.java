package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of CrossBridgeSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class CrossBridgeSystemKernels {
    private CrossBridgeSystemKernels() {}

    private static final MethodHandle H_XBRIDGE_BOND_FORCES = Sbx.h("sbx_xbridge_bond_forces",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** CrossBridgeSystem.bondForces (CrossBridgeSystem.java:58-142) -> sbx_xbridge_bond_forces. */
    public static void bondForces(FloatArray motorCoord, FloatArray motorUVec, FloatArray motorYVec, FloatArray motorBRotGam, FloatArray filCoord, FloatArray filUVec, FloatArray filYVec, FloatArray filBRotGam, FloatArray filSegLength, IntArray boundSeg, FloatArray bindArc, IntArray nucleotideState, FloatArray bondData, FloatArray xbParams) {
        Sbx.toDevice(motorCoord, motorUVec, motorYVec, motorBRotGam, filCoord, filUVec, filYVec, filBRotGam, filSegLength, boundSeg, bindArc, nucleotideState, bondData, xbParams);
        try {
            Sbx.check((int) H_XBRIDGE_BOND_FORCES.invokeExact(Sbx.ctx(), motorCoord.getSize() / 3, motorCoord.dev(), motorUVec.dev(), motorYVec.dev(), motorBRotGam.dev(), filCoord.getSize() / 3, filCoord.dev(), filUVec.dev(), filYVec.dev(), filBRotGam.dev(), filSegLength.dev(), boundSeg.dev(), bindArc.dev(), nucleotideState.dev(), bondData.dev(), xbParams.dev()), "sbx_xbridge_bond_forces");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(bondData);
    }

    private static final MethodHandle H_XBRIDGE_APPLY_HEAD_FORCE = Sbx.h("sbx_xbridge_apply_head_force",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS));

    /** CrossBridgeSystem.applyHeadForce (CrossBridgeSystem.java:145-157) -> sbx_xbridge_apply_head_force. */
    public static void applyHeadForce(FloatArray bondData, FloatArray bodyForceSum, FloatArray bodyTorqueSum, IntArray counts) {
        Sbx.toDevice(bondData, bodyForceSum, bodyTorqueSum);
        try {
            Sbx.check((int) H_XBRIDGE_APPLY_HEAD_FORCE.invokeExact(Sbx.ctx(), bodyForceSum.getSize() / 3, bondData.dev(), bodyForceSum.dev(), bodyTorqueSum.dev()), "sbx_xbridge_apply_head_force");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(bodyForceSum, bodyTorqueSum);
    }

    private static final MethodHandle H_XBRIDGE_REGISTER_FORCE_DOT = Sbx.h("sbx_xbridge_register_force_dot",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** CrossBridgeSystem.registerForceDot (CrossBridgeSystem.java:166-187) -> sbx_xbridge_register_force_dot. */
    public static void registerForceDot(FloatArray bondData, IntArray boundSeg, FloatArray forceDotFil, FloatArray forceMag, FloatArray forceDotHist, IntArray forceDotPlace, IntArray counts) {
        Sbx.toDevice(bondData, boundSeg, forceDotFil, forceMag, forceDotHist, forceDotPlace);
        try {
            Sbx.check((int) H_XBRIDGE_REGISTER_FORCE_DOT.invokeExact(Sbx.ctx(), boundSeg.getSize(), bondData.dev(), boundSeg.dev(), forceDotFil.dev(), forceMag.dev(), forceDotHist.dev(), forceDotPlace.dev()), "sbx_xbridge_register_force_dot");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(forceDotFil, forceMag, forceDotHist, forceDotPlace);
    }

    private static final MethodHandle H_CSR_SCAN = Sbx.h("sbx_csr_scan",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS));

    /** CrossBridgeSystem.csrScan (CrossBridgeSystem.java:198-205) -> sbx_csr_scan. */
    public static void csrScan(IntArray counts, IntArray segMotorCount, IntArray segMotorOffsets) {
        Sbx.toDevice(segMotorCount, segMotorOffsets);
        try {
            Sbx.check((int) H_CSR_SCAN.invokeExact(Sbx.ctx(), counts.get(3), segMotorCount.dev(), segMotorOffsets.dev()), "sbx_csr_scan");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(segMotorCount, segMotorOffsets);
    }

    private static final MethodHandle H_CSR_BUILD = Sbx.h("sbx_csr_build",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, JAVA_INT, ADDRESS, ADDRESS, ADDRESS));

    /** CrossBridgeSystem.csrChunkReduce (CrossBridgeSystem.java:260-276) -> sbx_csr_build. Note: the row counts (the histogram) of the keys recorded by csrChunkHistogram; csrScan then turns them into offsets. */
    public static void csrChunkReduce(IntArray counts, IntArray csrChunkParams, IntArray csrMatrix, IntArray segMotorCount) {
        CSR_BUILD.ensure(segMotorCount.getSize(), CSR_BUILD.nItems);
        Sbx.toDevice(CSR_BUILD.keys, segMotorCount, CSR_BUILD.offsets, CSR_BUILD.list);
        try {
            Sbx.check((int) H_CSR_BUILD.invokeExact(Sbx.ctx(), CSR_BUILD.keys.dev(), CSR_BUILD.nItems, segMotorCount.getSize(), segMotorCount.dev(), CSR_BUILD.offsets.dev(), CSR_BUILD.list.dev()), "sbx_csr_build");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(segMotorCount, CSR_BUILD.offsets, CSR_BUILD.list);
    }

    private static final MethodHandle H_CSR_BUILD_1 = Sbx.h("sbx_csr_build",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, JAVA_INT, ADDRESS, ADDRESS, ADDRESS));

    /** CrossBridgeSystem.csrChunkScatter (CrossBridgeSystem.java:278-298) -> sbx_csr_build. Note: the stable list: items in ascending index within each row, at the offsets csrScan wrote. */
    public static void csrChunkScatter(IntArray boundSeg, IntArray counts, IntArray csrChunkParams, IntArray segMotorOffsets, IntArray segMotorMyo, IntArray csrMatrix) {
        CSR_BUILD.ensure(segMotorOffsets.getSize() - 1, counts.get(0));
        Sbx.toDevice(boundSeg, CSR_BUILD.count, CSR_BUILD.offsets, segMotorMyo);
        try {
            Sbx.check((int) H_CSR_BUILD_1.invokeExact(Sbx.ctx(), boundSeg.dev(), counts.get(0), segMotorOffsets.getSize() - 1, CSR_BUILD.count.dev(), CSR_BUILD.offsets.dev(), segMotorMyo.dev()), "sbx_csr_build");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(CSR_BUILD.count, CSR_BUILD.offsets, segMotorMyo);
    }

    private static final MethodHandle H_XBRIDGE_SEG_GATHER = Sbx.h("sbx_xbridge_seg_gather",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** CrossBridgeSystem.segGather (CrossBridgeSystem.java:302-320) -> sbx_xbridge_seg_gather. */
    public static void segGather(IntArray segMotorOffsets, IntArray segMotorMyo, FloatArray bondData, FloatArray filForceSum, FloatArray filTorqueSum, IntArray counts) {
        Sbx.toDevice(segMotorOffsets, segMotorMyo, bondData, filForceSum, filTorqueSum);
        try {
            Sbx.check((int) H_XBRIDGE_SEG_GATHER.invokeExact(Sbx.ctx(), counts.get(3), segMotorOffsets.dev(), segMotorMyo.dev(), bondData.dev(), filForceSum.dev(), filTorqueSum.dev()), "sbx_xbridge_seg_gather");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(filForceSum, filTorqueSum);
    }

    /** CrossBridgeSystem.csrChunkZero (CrossBridgeSystem.java:232-237): its work runs in the build's last call. */
    public static void csrChunkZero(IntArray csrChunkParams, IntArray counts, IntArray csrMatrix) {
    }

    /** CrossBridgeSystem.csrChunkHistogram (CrossBridgeSystem.java:240-257): records its inputs; its work runs in the build's last call. */
    public static void csrChunkHistogram(IntArray boundSeg, IntArray counts, IntArray csrChunkParams, IntArray csrMatrix) {
        CSR_BUILD.record(boundSeg, counts.get(0), csrMatrix);
    }

    /** The keys of the chunked CSR build, recorded by csrChunkHistogram, and its scratch. */
    static final CsrBuild CSR_BUILD = new CsrBuild();

}
