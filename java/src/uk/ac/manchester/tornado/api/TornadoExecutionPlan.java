package uk.ac.manchester.tornado.api;

import softbox_b200.shim.DeviceArray;

/**
 * Stand-in: execute() replays the recorded System calls in order, each a downcall on the
 * library's one stream. Arrays passed with EVERY_EXECUTION are re-uploaded at every
 * execute(); FIRST_EXECUTION arrays are uploaded at their first device use; worker grids
 * are ignored (the library sizes its own launches).
 */
public final class TornadoExecutionPlan {
    private final ImmutableTaskGraph[] graphs;

    public TornadoExecutionPlan(ImmutableTaskGraph... graphs) { this.graphs = graphs; }

    public TornadoExecutionPlan withGridScheduler(GridScheduler scheduler) { return this; }

    public TornadoExecutionResult execute() {
        for (ImmutableTaskGraph g : graphs) {
            for (Object o : g.everyExecution) if (o instanceof DeviceArray d) d.markHostNewer();
            for (Runnable r : g.tasks) r.run();
        }
        return new TornadoExecutionResult();
    }
}
