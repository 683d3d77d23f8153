package softbox_b200.shim;

import uk.ac.manchester.tornado.api.types.arrays.IntArray;

/**
 * The chunked grid build of the reference (gridChunkZero, gridChunkHistogram,
 * gridChunkReduce, gridScanLocal, gridScanChunks, gridScanAdd, gridChunkScatter) runs in the
 * library as one stable counting sort (sbx_grid_build). gridChunkHistogram records its
 * inputs here; gridScanAdd, the first call that holds every output array, runs the build.
 */
final class GridBuild {
    IntArray bodyCell;
    IntArray counts;
    int cap;

    void record(IntArray bodyCell, IntArray counts) {
        this.bodyCell = bodyCell;
        this.counts = counts;
        this.cap = bodyCell.getSize();
    }
}
