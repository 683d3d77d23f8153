package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of MotorJointSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class MotorJointSystemKernels {
    private MotorJointSystemKernels() {}

    private static final MethodHandle H_MOTOR_JOINTS = Sbx.h("sbx_motor_joints",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** MotorJointSystem.joints (MotorJointSystem.java:72-197) -> sbx_motor_joints. */
    public static void joints(FloatArray coord, FloatArray uVec, FloatArray segLength, FloatArray bTransGam, FloatArray bRotGam, FloatArray forceSum, FloatArray torqueSum, IntArray nucleotideState, FloatArray jointParams, IntArray counts) {
        Sbx.toDevice(coord, uVec, segLength, bTransGam, bRotGam, forceSum, torqueSum, nucleotideState, jointParams);
        try {
            Sbx.check((int) H_MOTOR_JOINTS.invokeExact(Sbx.ctx(), coord.getSize() / 3, coord.dev(), uVec.dev(), segLength.dev(), bTransGam.dev(), bRotGam.dev(), forceSum.dev(), torqueSum.dev(), nucleotideState.dev(), jointParams.dev()), "sbx_motor_joints");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(forceSum, torqueSum);
    }

}
