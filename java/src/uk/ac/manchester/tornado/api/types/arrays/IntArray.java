package uk.ac.manchester.tornado.api.types.arrays;

import java.lang.foreign.Arena;
import java.lang.foreign.MemorySegment;

import softbox_b200.shim.DeviceArray;
import softbox_b200.shim.SbxAccess;

import static java.lang.foreign.ValueLayout.JAVA_INT;

/**
 * Stand-in for TornadoVM's IntArray over libsoftbox_b200: the host copy is an off-heap
 * segment (what get/set touch, as before), the device copy a library allocation (what the
 * System downcalls receive). The copies are kept coherent lazily: get/set pull a newer
 * device copy first; a downcall uploads a newer host copy first.
 */
public final class IntArray implements DeviceArray {
    private final int size;
    private final MemorySegment host;
    private MemorySegment dev;
    private boolean hostNewer = true;     // nothing on the device yet
    private boolean deviceNewer = false;

    public IntArray(int numElements) {
        size = numElements;
        host = Arena.global().allocate(4L * Math.max(1, numElements), 16);
    }

    public static IntArray fromElements(int... values) {
        IntArray a = new IntArray(values.length);
        for (int i = 0; i < values.length; i++) a.set(i, values[i]);
        return a;
    }

    public int getSize() { return size; }

    public int get(int i) {
        if (deviceNewer) syncToHost();
        return host.getAtIndex(JAVA_INT, i);
    }

    public void set(int i, int v) {
        if (deviceNewer) syncToHost();
        host.setAtIndex(JAVA_INT, i, v);
        hostNewer = true;
    }

    public void init(int v) {
        if (deviceNewer) syncToHost();
        for (int i = 0; i < size; i++) host.setAtIndex(JAVA_INT, i, v);
        hostNewer = true;
    }

    public void clear() { init((int) 0); }

    @Override
    public MemorySegment dev() {
        syncToDevice();
        return dev;
    }

    @Override
    public void syncToDevice() {
        if (dev == null) dev = SbxAccess.alloc(4L * Math.max(1, size));
        if (hostNewer) {
            SbxAccess.upload(dev, host, 4L * size);
            hostNewer = false;
        }
    }

    @Override
    public void markDeviceNewer() {
        if (dev != null) deviceNewer = true;
    }

    @Override
    public void syncToHost() {
        if (deviceNewer) {
            SbxAccess.download(host, dev, 4L * size);
            deviceNewer = false;
        }
    }

    @Override
    public void markHostNewer() {
        if (deviceNewer) syncToHost();
        hostNewer = true;
    }
}
