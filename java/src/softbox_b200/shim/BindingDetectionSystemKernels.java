package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of BindingDetectionSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class BindingDetectionSystemKernels {
    private BindingDetectionSystemKernels() {}

    private static final MethodHandle H_BINDING_GRID_REACHABLE = Sbx.h("sbx_binding_grid_reachable",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_INT));

    /** BindingDetectionSystem.gridReachable (BindingDetectionSystem.java:143-228) -> sbx_binding_grid_reachable. */
    public static void gridReachable(FloatArray head, FloatArray uVec, FloatArray rodUVec, FloatArray segEnd1, FloatArray segEnd2, FloatArray gridParams, IntArray gridDims, IntArray gridCellOffsets, IntArray gridCellContents, IntArray ownerStore, IntArray ownerSlot, IntArray motorReachSeg, IntArray motorReachCount, FloatArray kinParams, IntArray counts) {
        Sbx.toDevice(head, uVec, rodUVec, segEnd1, segEnd2, gridParams, gridDims, gridCellOffsets, gridCellContents, ownerStore, ownerSlot, motorReachSeg, motorReachCount, kinParams);
        try {
            Sbx.check((int) H_BINDING_GRID_REACHABLE.invokeExact(Sbx.ctx(), head.dev(), uVec.dev(), rodUVec.dev(), segEnd1.getSize() / 3, segEnd1.dev(), segEnd2.dev(), gridParams.dev(), gridDims.dev(), gridCellOffsets.dev(), gridCellContents.dev(), ownerStore.dev(), ownerSlot.dev(), motorReachSeg.dev(), motorReachCount.dev(), kinParams.dev(), counts.get(0)), "sbx_binding_grid_reachable");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(motorReachSeg, motorReachCount);
    }

    private static final MethodHandle H_BINDING_BIND_NEAREST = Sbx.h("sbx_binding_bind_nearest",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_INT));

    /** BindingDetectionSystem.bindNearest (BindingDetectionSystem.java:356-389) -> sbx_binding_bind_nearest. */
    public static void bindNearest(FloatArray head, FloatArray uVec, FloatArray rodUVec, FloatArray segEnd1, FloatArray segEnd2, IntArray motorCandSeg, IntArray motorCandCount, IntArray boundSeg, FloatArray bindArc, FloatArray kinParams, IntArray counts) {
        Sbx.toDevice(head, uVec, rodUVec, segEnd1, segEnd2, motorCandSeg, motorCandCount, boundSeg, bindArc, kinParams);
        try {
            Sbx.check((int) H_BINDING_BIND_NEAREST.invokeExact(Sbx.ctx(), head.dev(), uVec.dev(), rodUVec.dev(), segEnd1.getSize() / 3, segEnd1.dev(), segEnd2.dev(), motorCandSeg.dev(), motorCandCount.dev(), boundSeg.dev(), bindArc.dev(), kinParams.dev(), counts.get(0)), "sbx_binding_bind_nearest");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(boundSeg, bindArc);
    }

}
