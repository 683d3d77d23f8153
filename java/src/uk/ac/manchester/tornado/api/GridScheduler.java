package uk.ac.manchester.tornado.api;

import java.util.HashMap;
import java.util.Map;

/** Stand-in: records worker grids by task name; the library sizes its own launches. */
public final class GridScheduler {
    private final Map<String, WorkerGrid> grids = new HashMap<>();

    public void addWorkerGrid(String taskName, WorkerGrid grid) { grids.put(taskName, grid); }

    public WorkerGrid get(String taskName) { return grids.get(taskName); }
}
