package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of MotorStore's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class MotorStoreKernels {
    private MotorStoreKernels() {}

    private static final MethodHandle H_MOTOR_PUBLISH_HEAD = Sbx.h("sbx_motor_publish_head",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** MotorStore.publishHeadFromBody (MotorStore.java:300-314) -> sbx_motor_publish_head. */
    public static void publishHeadFromBody(FloatArray bodyCoord, FloatArray bodyUVec, FloatArray bodySegLength, FloatArray head, FloatArray uVec, FloatArray rodUVec, IntArray counts) {
        Sbx.toDevice(bodyCoord, bodyUVec, bodySegLength, head, uVec, rodUVec);
        try {
            Sbx.check((int) H_MOTOR_PUBLISH_HEAD.invokeExact(Sbx.ctx(), head.getSize() / 3, bodyCoord.dev(), bodyUVec.dev(), bodySegLength.dev(), head.dev(), uVec.dev(), rodUVec.dev()), "sbx_motor_publish_head");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(head, uVec, rodUVec);
    }

    private static final MethodHandle H_MOTOR_PUBLISH = Sbx.h("sbx_motor_publish",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** MotorStore.publishToBodyView (MotorStore.java:326-347) -> sbx_motor_publish. */
    public static void publishToBodyView(FloatArray head, FloatArray reach, FloatArray center, FloatArray boundingRadius, IntArray ownerStore, IntArray ownerSlot, IntArray publishParams, IntArray counts) {
        Sbx.toDevice(head, reach, center, boundingRadius, ownerStore, ownerSlot, publishParams);
        try {
            Sbx.check((int) H_MOTOR_PUBLISH.invokeExact(Sbx.ctx(), head.getSize() / 3, head.dev(), reach.dev(), center.getSize() / 3, center.dev(), boundingRadius.dev(), ownerStore.dev(), ownerSlot.dev(), publishParams.dev()), "sbx_motor_publish");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(center, boundingRadius, ownerStore, ownerSlot);
    }

}
