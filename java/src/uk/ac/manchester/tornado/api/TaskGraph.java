package uk.ac.manchester.tornado.api;

import java.util.ArrayList;
import java.util.List;

import uk.ac.manchester.tornado.api.common.TornadoFunctions;
import uk.ac.manchester.tornado.api.enums.DataTransferMode;

/**
 * Stand-in for TornadoVM's TaskGraph (generated by java/gen_shim.py): records the
 * tasks, whose bodies are the System methods (now libsoftbox_b200 downcalls), and the
 * arrays to re-upload at every execute(); snapshot() freezes the list.
 */
public final class TaskGraph {
    private final String name;
    private final List<Runnable> tasks = new ArrayList<>();
    private final List<Object> everyExecution = new ArrayList<>();

    public TaskGraph(String name) { this.name = name; }

    public String getTaskGraphName() { return name; }

    public TaskGraph transferToDevice(DataTransferMode mode, Object... arrays) {
        if (mode == DataTransferMode.EVERY_EXECUTION) everyExecution.addAll(List.of(arrays));
        return this;
    }

    public TaskGraph transferToHost(DataTransferMode mode, Object... arrays) { return this; }

    public ImmutableTaskGraph snapshot() { return new ImmutableTaskGraph(tasks, everyExecution); }

    public <T1> TaskGraph task(String id, TornadoFunctions.Task1<T1> code, T1 a1) {
        tasks.add(() -> code.apply(a1));
        return this;
    }

    public <T1, T2> TaskGraph task(String id, TornadoFunctions.Task2<T1, T2> code, T1 a1, T2 a2) {
        tasks.add(() -> code.apply(a1, a2));
        return this;
    }

    public <T1, T2, T3> TaskGraph task(String id, TornadoFunctions.Task3<T1, T2, T3> code, T1 a1, T2 a2, T3 a3) {
        tasks.add(() -> code.apply(a1, a2, a3));
        return this;
    }

    public <T1, T2, T3, T4> TaskGraph task(String id, TornadoFunctions.Task4<T1, T2, T3, T4> code, T1 a1, T2 a2, T3 a3, T4 a4) {
        tasks.add(() -> code.apply(a1, a2, a3, a4));
        return this;
    }

    public <T1, T2, T3, T4, T5> TaskGraph task(String id, TornadoFunctions.Task5<T1, T2, T3, T4, T5> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5));
        return this;
    }

    public <T1, T2, T3, T4, T5, T6> TaskGraph task(String id, TornadoFunctions.Task6<T1, T2, T3, T4, T5, T6> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5, a6));
        return this;
    }

    public <T1, T2, T3, T4, T5, T6, T7> TaskGraph task(String id, TornadoFunctions.Task7<T1, T2, T3, T4, T5, T6, T7> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6, T7 a7) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5, a6, a7));
        return this;
    }

    public <T1, T2, T3, T4, T5, T6, T7, T8> TaskGraph task(String id, TornadoFunctions.Task8<T1, T2, T3, T4, T5, T6, T7, T8> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6, T7 a7, T8 a8) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5, a6, a7, a8));
        return this;
    }

    public <T1, T2, T3, T4, T5, T6, T7, T8, T9> TaskGraph task(String id, TornadoFunctions.Task9<T1, T2, T3, T4, T5, T6, T7, T8, T9> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6, T7 a7, T8 a8, T9 a9) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5, a6, a7, a8, a9));
        return this;
    }

    public <T1, T2, T3, T4, T5, T6, T7, T8, T9, T10> TaskGraph task(String id, TornadoFunctions.Task10<T1, T2, T3, T4, T5, T6, T7, T8, T9, T10> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6, T7 a7, T8 a8, T9 a9, T10 a10) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5, a6, a7, a8, a9, a10));
        return this;
    }

    public <T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11> TaskGraph task(String id, TornadoFunctions.Task11<T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6, T7 a7, T8 a8, T9 a9, T10 a10, T11 a11) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11));
        return this;
    }

    public <T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12> TaskGraph task(String id, TornadoFunctions.Task12<T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6, T7 a7, T8 a8, T9 a9, T10 a10, T11 a11, T12 a12) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12));
        return this;
    }

    public <T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12, T13> TaskGraph task(String id, TornadoFunctions.Task13<T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12, T13> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6, T7 a7, T8 a8, T9 a9, T10 a10, T11 a11, T12 a12, T13 a13) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13));
        return this;
    }

    public <T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12, T13, T14> TaskGraph task(String id, TornadoFunctions.Task14<T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12, T13, T14> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6, T7 a7, T8 a8, T9 a9, T10 a10, T11 a11, T12 a12, T13 a13, T14 a14) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14));
        return this;
    }

    public <T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12, T13, T14, T15> TaskGraph task(String id, TornadoFunctions.Task15<T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12, T13, T14, T15> code, T1 a1, T2 a2, T3 a3, T4 a4, T5 a5, T6 a6, T7 a7, T8 a8, T9 a9, T10 a10, T11 a11, T12 a12, T13 a13, T14 a14, T15 a15) {
        tasks.add(() -> code.apply(a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14, a15));
        return this;
    }

}
