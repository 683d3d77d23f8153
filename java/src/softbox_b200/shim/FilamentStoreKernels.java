package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of FilamentStore's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class FilamentStoreKernels {
    private FilamentStoreKernels() {}

    private static final MethodHandle H_FILAMENT_PUBLISH = Sbx.h("sbx_filament_publish",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** FilamentStore.publishToBodyView (FilamentStore.java:275-295) -> sbx_filament_publish. */
    public static void publishToBodyView(FloatArray coord, FloatArray segLength, FloatArray center, FloatArray boundingRadius, IntArray ownerStore, IntArray ownerSlot, FloatArray viewParams, IntArray counts) {
        Sbx.toDevice(coord, segLength, center, boundingRadius, ownerStore, ownerSlot, viewParams);
        try {
            Sbx.check((int) H_FILAMENT_PUBLISH.invokeExact(Sbx.ctx(), coord.getSize() / 3, coord.dev(), segLength.dev(), center.getSize() / 3, center.dev(), boundingRadius.dev(), ownerStore.dev(), ownerSlot.dev(), viewParams.dev(), MemorySegment.NULL), "sbx_filament_publish");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(center, boundingRadius, ownerStore, ownerSlot);
    }

    private static final MethodHandle H_FILAMENT_PUBLISH_1 = Sbx.h("sbx_filament_publish",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** FilamentStore.publishToBodyView (FilamentStore.java:306-328) -> sbx_filament_publish. */
    public static void publishToBodyView(FloatArray coord, FloatArray segLength, FloatArray center, FloatArray boundingRadius, IntArray ownerStore, IntArray ownerSlot, FloatArray viewParams, IntArray counts, IntArray filState) {
        Sbx.toDevice(coord, segLength, center, boundingRadius, ownerStore, ownerSlot, viewParams, filState);
        try {
            Sbx.check((int) H_FILAMENT_PUBLISH_1.invokeExact(Sbx.ctx(), coord.getSize() / 3, coord.dev(), segLength.dev(), center.getSize() / 3, center.dev(), boundingRadius.dev(), ownerStore.dev(), ownerSlot.dev(), viewParams.dev(), filState.dev()), "sbx_filament_publish");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(center, boundingRadius, ownerStore, ownerSlot);
    }

}
