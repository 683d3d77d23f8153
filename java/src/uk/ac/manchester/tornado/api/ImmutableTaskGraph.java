package uk.ac.manchester.tornado.api;

import java.util.List;

/** Stand-in: the frozen task list of a TaskGraph (TaskGraph.snapshot()). */
public final class ImmutableTaskGraph {
    final List<Runnable> tasks;
    final List<Object> everyExecution;

    ImmutableTaskGraph(List<Runnable> tasks, List<Object> everyExecution) {
        this.tasks = List.copyOf(tasks);
        this.everyExecution = List.copyOf(everyExecution);
    }
}
