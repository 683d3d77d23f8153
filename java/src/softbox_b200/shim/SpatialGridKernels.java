package softbox_b200.shim;

import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.MethodHandle;

import uk.ac.manchester.tornado.api.types.arrays.FloatArray;
import uk.ac.manchester.tornado.api.types.arrays.IntArray;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;

/** Downcall bodies of SpatialGrid's kernels (generated by java/gen_shim.py). Each method has the
 *  reference method's Java signature; its body moves the arguments' current contents to the
 *  device, calls the C entry point on the shim's context and marks the arrays device-newer. */
public final class SpatialGridKernels {
    private SpatialGridKernels() {}

    private static final MethodHandle H_GRID_BODY_CELL = Sbx.h("sbx_grid_body_cell",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));

    /** SpatialGrid.bodyCell (SpatialGrid.java:51-75) -> sbx_grid_body_cell. */
    public static void bodyCell(FloatArray center, FloatArray gridParams, IntArray gridDims, IntArray counts, IntArray bodyCell) {
        Sbx.toDevice(center, gridParams, gridDims, counts, bodyCell);
        try {
            Sbx.check((int) H_GRID_BODY_CELL.invokeExact(Sbx.ctx(), center.getSize() / 3, center.dev(), gridParams.dev(), gridDims.dev(), counts.dev(), bodyCell.dev()), "sbx_grid_body_cell");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        Sbx.written(bodyCell);
    }

    private static final MethodHandle H_GRID_BUILD = Sbx.h("sbx_grid_build",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_INT));

    /** SpatialGrid.gridScanAdd (SpatialGrid.java:137-160) -> sbx_grid_build. Note: the chunked build (gridChunkZero/Histogram/Reduce, gridScanLocal/Chunks/Add, gridChunkScatter) runs as one stable counting sort here, over the bodyCell / counts recorded by gridChunkHistogram; cellCount is then reset as the scan's write cursor. */
    public static void gridScanAdd(IntArray gridDims, IntArray gridCellOffsets, IntArray gridCellContents, IntArray cellCount, IntArray chunkSum) {
        Sbx.toDevice(GRID_BUILD.bodyCell, GRID_BUILD.counts, cellCount, chunkSum, gridCellOffsets, gridCellContents);
        try {
            Sbx.check((int) H_GRID_BUILD.invokeExact(Sbx.ctx(), GRID_BUILD.cap, GRID_BUILD.bodyCell.dev(), GRID_BUILD.counts.dev(), gridDims.get(3), cellCount.dev(), chunkSum.dev(), gridCellOffsets.dev(), gridCellContents.dev(), gridCellContents.getSize()), "sbx_grid_build");
        } catch (Throwable t) {
            throw Sbx.rethrow(t);
        }
        // the chunked reference leaves cellCount zero (its scan's write cursor, unused by
        // the chunk scatter)
        SbxAccess.memset(cellCount.dev(), 0, 4L * cellCount.getSize());
        Sbx.written(cellCount, chunkSum, gridCellOffsets, gridCellContents);
    }

    /** SpatialGrid.gridChunkZero (SpatialGrid.java:237-244): its work runs in the build's last call. */
    public static void gridChunkZero(IntArray chunkParams, IntArray gridDims, IntArray chunkCellCount) {
    }

    /** SpatialGrid.gridChunkHistogram (SpatialGrid.java:248-273): records its inputs; its work runs in the build's last call. */
    public static void gridChunkHistogram(IntArray bodyCell, IntArray counts, IntArray chunkParams, IntArray gridDims, IntArray chunkCellCount) {
        GRID_BUILD.record(bodyCell, counts);
    }

    /** SpatialGrid.gridChunkReduce (SpatialGrid.java:278-296): its work runs in the build's last call. */
    public static void gridChunkReduce(IntArray gridDims, IntArray chunkParams, IntArray chunkCellCount, IntArray cellCount) {
    }

    /** SpatialGrid.gridScanLocal (SpatialGrid.java:99-117): its work runs in the build's last call. */
    public static void gridScanLocal(IntArray gridDims, IntArray cellCount, IntArray gridCellOffsets, IntArray chunkSum) {
    }

    /** SpatialGrid.gridScanChunks (SpatialGrid.java:121-133): its work runs in the build's last call. */
    public static void gridScanChunks(IntArray gridDims, IntArray chunkSum) {
    }

    /** SpatialGrid.gridChunkScatter (SpatialGrid.java:302-331): its work runs in the build's last call. */
    public static void gridChunkScatter(IntArray bodyCell, IntArray counts, IntArray chunkParams, IntArray gridDims, IntArray gridCellOffsets, IntArray gridCellContents, IntArray chunkCellCount) {
    }

    /** The inputs of the chunked grid build, recorded by gridChunkHistogram. */
    static final GridBuild GRID_BUILD = new GridBuild();

}
