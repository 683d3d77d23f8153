package softbox_b200.shim;

import uk.ac.manchester.tornado.api.types.arrays.IntArray;

/**
 * The chunked CSR-inverse build of the reference (csrChunkZero, csrChunkHistogram,
 * csrChunkReduce, csrScan, csrChunkScatter). csrChunkHistogram records the keys;
 * csrChunkReduce writes the row counts (sbx_csr_build into scratch offsets and list);
 * csrScan turns them into offsets (sbx_csr_scan, which also clears the counts as the
 * reference's write cursor); csrChunkScatter writes the stable list (sbx_csr_build with the
 * counts and offsets in scratch: the same offsets csrScan wrote). The builds of one step run
 * one after another, so one scratch set serves them all; it grows to the largest build.
 */
final class CsrBuild {
    IntArray keys;
    int nItems;
    IntArray count = new IntArray(1);
    IntArray offsets = new IntArray(2);
    IntArray list = new IntArray(1);

    void record(IntArray keys, int nItems, IntArray matrix) {
        this.keys = keys;
        this.nItems = nItems;
    }

    void ensure(int nRows, int items) {
        if (count.getSize() < nRows) count = new IntArray(nRows);
        if (offsets.getSize() < nRows + 1) offsets = new IntArray(nRows + 1);
        if (list.getSize() < Math.max(1, items)) list = new IntArray(Math.max(1, items));
    }
}
