package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of DeflectionSupport's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class DeflectionSupportKernels {
    private DeflectionSupportKernels() {}

    private static final MethodHandle H_DEFLECTION_SEED_ACCUMULATORS = Sbx.h("sbx_deflection_seed_accumulators",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** DeflectionSupport.seedAccumulators (DeflectionSupport.java:24-33) -> sbx_deflection_seed_accumulators. */
    public static void seedAccumulators(FloatArray forceSum, FloatArray torqueSum, FloatArray extForce, IntArray counts) {
        Sbx.toDevice(forceSum, torqueSum, extForce, counts);
        try {
            Sbx.check((int) H_DEFLECTION_SEED_ACCUMULATORS.invokeExact(Sbx.ctx(), forceSum.getSize() / 3, forceSum.dev(), torqueSum.dev(), extForce.dev(), counts.dev()), "sbx_deflection_seed_accumulators");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(forceSum, torqueSum);
    }

    private static final MethodHandle H_DEFLECTION_PIN_ENDPOINTS = Sbx.h("sbx_deflection_pin_endpoints",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS));

    /** DeflectionSupport.pinEndpoints (DeflectionSupport.java:40-58) -> sbx_deflection_pin_endpoints. */
    public static void pinEndpoints(FloatArray coord, FloatArray uVec, FloatArray segLength, IntArray pinSeg, IntArray pinEnd, FloatArray pinAnchor, IntArray counts) {
        Sbx.toDevice(coord, uVec, segLength, pinSeg, pinEnd, pinAnchor);
        try {
            Sbx.check((int) H_DEFLECTION_PIN_ENDPOINTS.invokeExact(Sbx.ctx(), coord.getSize() / 3, coord.dev(), uVec.dev(), segLength.dev(), pinSeg.getSize(), pinSeg.dev(), pinEnd.dev(), pinAnchor.dev()), "sbx_deflection_pin_endpoints");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(coord);
    }

}
