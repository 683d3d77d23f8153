package softbox_b200.shim;

import java.lang.foreign.MemorySegment;

/** The memory operations the array stand-ins (in TornadoVM's package) need from Sbx. */
public final class SbxAccess {
    private SbxAccess() {}

    public static MemorySegment alloc(long bytes) { return Sbx.deviceAlloc(bytes); }

    public static void upload(MemorySegment dev, MemorySegment host, long bytes) { Sbx.upload(dev, host, bytes); }

    public static void download(MemorySegment host, MemorySegment dev, long bytes) { Sbx.download(host, dev, bytes); }

    public static void memset(MemorySegment dev, int value, long bytes) { Sbx.memset(dev, value, bytes); }
}
