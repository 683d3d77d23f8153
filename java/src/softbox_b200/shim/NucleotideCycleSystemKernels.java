package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of NucleotideCycleSystem's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class NucleotideCycleSystemKernels {
    private NucleotideCycleSystemKernels() {}

    private static final MethodHandle H_NUCLEOTIDE_CYCLE = Sbx.h("sbx_nucleotide_cycle",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** NucleotideCycleSystem.cycle (NucleotideCycleSystem.java:33-69) -> sbx_nucleotide_cycle. */
    public static void cycle(IntArray nucleotideState, IntArray boundSeg, FloatArray forceDotHist, FloatArray nucParams, IntArray counts) {
        Sbx.toDevice(nucleotideState, boundSeg, forceDotHist, nucParams, counts);
        try {
            Sbx.check((int) H_NUCLEOTIDE_CYCLE.invokeExact(Sbx.ctx(), nucleotideState.getSize(), nucleotideState.dev(), boundSeg.dev(), forceDotHist.dev(), nucParams.dev(), counts.dev()), "sbx_nucleotide_cycle");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(nucleotideState);
    }

    private static final MethodHandle H_NUCLEOTIDE_RELEASE = Sbx.h("sbx_nucleotide_release",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** NucleotideCycleSystem.catchSlipRelease (NucleotideCycleSystem.java:77-134) -> sbx_nucleotide_release. */
    public static void catchSlipRelease(IntArray boundSeg, FloatArray forceDotFil, FloatArray forceMag, IntArray cooldown, IntArray stats, IntArray capStats, FloatArray kinParams, IntArray counts) {
        Sbx.toDevice(boundSeg, forceDotFil, forceMag, cooldown, stats, capStats, kinParams, counts);
        try {
            Sbx.check((int) H_NUCLEOTIDE_RELEASE.invokeExact(Sbx.ctx(), boundSeg.getSize(), boundSeg.dev(), forceDotFil.dev(), forceMag.dev(), cooldown.dev(), stats.dev(), capStats.dev(), kinParams.dev(), counts.dev()), "sbx_nucleotide_release");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(boundSeg, cooldown, stats, capStats);
    }

}
