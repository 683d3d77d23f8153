package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of DragTensorSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class DragTensorSystemKernels {
    private DragTensorSystemKernels() {}

    private static final MethodHandle H_DRAG_RUN_FILAMENT = Sbx.h("sbx_drag_run_filament",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_DOUBLE, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** DragTensorSystem.runFilament (DragTensorSystem.java:71-97) -> sbx_drag_run_filament. Note: DragTensorSystem.run(FilamentStore s) delegates with s's arrays and Constants.aeta. */
    public static void runFilament(FloatArray segLength, IntArray monomerCount, IntArray end1NbrSlot, IntArray end2NbrSlot, FloatArray bTransGam, FloatArray bRotGam, FloatArray bTransDiff, FloatArray bRotDiff, double aeta) {
        Sbx.toDevice(monomerCount, end1NbrSlot, end2NbrSlot, segLength, bTransGam, bRotGam, bTransDiff, bRotDiff);
        try {
            Sbx.check((int) H_DRAG_RUN_FILAMENT.invokeExact(Sbx.ctx(), segLength.getSize(), monomerCount.dev(), end1NbrSlot.dev(), end2NbrSlot.dev(), aeta, segLength.dev(), bTransGam.dev(), bRotGam.dev(), bTransDiff.dev(), bRotDiff.dev()), "sbx_drag_run_filament");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(segLength, bTransGam, bRotGam, bTransDiff, bRotDiff);
    }

    private static final MethodHandle H_DRAG_RUN_MOTOR = Sbx.h("sbx_drag_run_motor",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, JAVA_DOUBLE, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** DragTensorSystem.runMotor (DragTensorSystem.java:105-122) -> sbx_drag_run_motor. Note: DragTensorSystem.run(MotorStore mot) delegates with mot.body's arrays and Constants.aeta. */
    public static void runMotor(FloatArray segLength, FloatArray bTransGam, FloatArray bRotGam, FloatArray bTransDiff, FloatArray bRotDiff, double aeta) {
        Sbx.toDevice(segLength, bTransGam, bRotGam, bTransDiff, bRotDiff);
        try {
            Sbx.check((int) H_DRAG_RUN_MOTOR.invokeExact(Sbx.ctx(), segLength.getSize() / 3, aeta, segLength.dev(), bTransGam.dev(), bRotGam.dev(), bTransDiff.dev(), bRotDiff.dev()), "sbx_drag_run_motor");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(segLength, bTransGam, bRotGam, bTransDiff, bRotDiff);
    }

}
