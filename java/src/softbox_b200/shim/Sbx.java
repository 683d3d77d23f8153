package softbox_b200.shim;

import java.lang.foreign.Arena;
import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.Linker;
import java.lang.foreign.MemorySegment;
import java.lang.foreign.SymbolLookup;
import java.lang.invoke.MethodHandle;
import java.nio.file.Path;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_INT;
import static java.lang.foreign.ValueLayout.JAVA_LONG;

/**
 * The Java side of libsoftbox_b200.so: loads the library through the Foreign Function &
 * Memory API (java.lang.foreign, final in JDK 22, preview in 21 with --enable-preview),
 * owns the one context every downcall runs on (one CUDA stream, calls in program order),
 * and moves array contents between a stand-in array's host segment and its device
 * allocation on demand.
 *
 * Library path: the SOFTBOX_B200_LIB environment variable, else the system property
 * softbox_b200.lib. Every failing status raises SbxException with the library's message.
 */
public final class Sbx {
    private Sbx() {}

    private static final Linker LINKER = Linker.nativeLinker();
    private static final SymbolLookup LIB = SymbolLookup.libraryLookup(Path.of(libraryPath()), Arena.global());

    private static String libraryPath() {
        String p = System.getenv("SOFTBOX_B200_LIB");
        if (p == null) p = System.getProperty("softbox_b200.lib");
        if (p == null) throw new IllegalStateException("set SOFTBOX_B200_LIB to libsoftbox_b200.so");
        return p;
    }

    /** A downcall handle for an exported function of the library. */
    public static MethodHandle h(String name, FunctionDescriptor fd) {
        MemorySegment fn = LIB.find(name).orElseThrow(() -> new UnsatisfiedLinkError("libsoftbox_b200: " + name));
        return LINKER.downcallHandle(fn, fd);
    }

    private static final MethodHandle CTX_CREATE = h("sbx_ctx_create", FunctionDescriptor.of(JAVA_INT, JAVA_INT, ADDRESS, ADDRESS));
    private static final MethodHandle LAST_ERROR = h("sbx_ctx_last_error", FunctionDescriptor.of(ADDRESS, ADDRESS));
    private static final MethodHandle SYNC = h("sbx_ctx_sync", FunctionDescriptor.of(JAVA_INT, ADDRESS));
    private static final MethodHandle MALLOC = h("sbx_malloc", FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_LONG, ADDRESS));
    private static final MethodHandle FREE = h("sbx_free", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
    private static final MethodHandle UPLOAD = h("sbx_upload", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_LONG));
    private static final MethodHandle DOWNLOAD = h("sbx_download", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_LONG));
    private static final MethodHandle MEMSET = h("sbx_memset", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, JAVA_LONG));

    private static final MemorySegment CTX = createContext();

    private static MemorySegment createContext() {
        try (Arena a = Arena.ofConfined()) {
            MemorySegment out = a.allocate(ADDRESS);
            int st = (int) CTX_CREATE.invokeExact(Integer.getInteger("softbox_b200.device", 0), MemorySegment.NULL, out);
            if (st != 0) throw new SbxException(st, "sbx_ctx_create");
            return out.get(ADDRESS, 0);
        } catch (SbxException e) {
            throw e;
        } catch (Throwable t) {
            throw new ExceptionInInitializerError(t);
        }
    }

    /** The context every downcall of the shim runs on. */
    public static MemorySegment ctx() { return CTX; }

    /** The library's message for the last failing call on the context. */
    public static String lastError() {
        try {
            MemorySegment s = (MemorySegment) LAST_ERROR.invokeExact(CTX);
            return s.reinterpret(4096).getString(0);
        } catch (Throwable t) {
            return "(no message)";
        }
    }

    public static void check(int status, String what) {
        if (status != 0) throw new SbxException(status, what + ": " + lastError());
    }

    public static RuntimeException rethrow(Throwable t) {
        if (t instanceof RuntimeException r) return r;
        if (t instanceof Error e) throw e;
        return new RuntimeException(t);
    }

    /** Waits for the context's stream (and reports an out-of-range input a kernel skipped). */
    public static void sync() {
        try { check((int) SYNC.invokeExact(CTX), "sbx_ctx_sync"); } catch (Throwable t) { throw rethrow(t); }
    }

    static MemorySegment deviceAlloc(long bytes) {
        try (Arena a = Arena.ofConfined()) {
            MemorySegment out = a.allocate(ADDRESS);
            check((int) MALLOC.invokeExact(CTX, bytes, out), "sbx_malloc");
            return out.get(ADDRESS, 0);
        } catch (Throwable t) { throw rethrow(t); }
    }

    static void deviceFree(MemorySegment dev) {
        try { check((int) FREE.invokeExact(CTX, dev), "sbx_free"); } catch (Throwable t) { throw rethrow(t); }
    }

    static void upload(MemorySegment dev, MemorySegment host, long bytes) {
        try { check((int) UPLOAD.invokeExact(CTX, dev, host, bytes), "sbx_upload"); } catch (Throwable t) { throw rethrow(t); }
    }

    /** Device-to-host copy; waits for the stream, so the host segment is valid on return. */
    static void download(MemorySegment host, MemorySegment dev, long bytes) {
        try { check((int) DOWNLOAD.invokeExact(CTX, host, dev, bytes), "sbx_download"); } catch (Throwable t) { throw rethrow(t); }
    }

    static void memset(MemorySegment dev, int value, long bytes) {
        try { check((int) MEMSET.invokeExact(CTX, dev, value, bytes), "sbx_memset"); } catch (Throwable t) { throw rethrow(t); }
    }

    /** Before a downcall: every argument array's device copy holds its current contents. */
    public static void toDevice(DeviceArray... arrays) {
        for (DeviceArray a : arrays) if (a != null) a.syncToDevice();
    }

    /** After a downcall: the arguments' device copies are the current ones (a host read pulls them). */
    public static void written(DeviceArray... arrays) {
        for (DeviceArray a : arrays) if (a != null) a.markDeviceNewer();
    }
}
