package uk.ac.manchester.tornado.api;

/** Stand-in for TornadoVM's one-dimensional worker grid. */
public final class WorkerGrid1D extends WorkerGrid {
    public WorkerGrid1D(long globalX) { global = new long[]{globalX, 1, 1}; }
}
