package uk.ac.manchester.tornado.api;

/** Stand-in for TornadoVM's worker grid: global and local sizes, recorded only. */
public class WorkerGrid {
    protected long[] global = {1, 1, 1};
    protected long[] local = {1, 1, 1};

    public void setLocalWork(long x, long y, long z) { local = new long[]{x, y, z}; }

    public void setGlobalWork(long x, long y, long z) { global = new long[]{x, y, z}; }
}
