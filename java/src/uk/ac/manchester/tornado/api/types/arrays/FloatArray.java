package uk.ac.manchester.tornado.api.types.arrays;

import java.lang.foreign.Arena;
import java.lang.foreign.MemorySegment;

import softbox_b200.shim.DeviceArray;
import softbox_b200.shim.SbxAccess;

import static java.lang.foreign.ValueLayout.JAVA_FLOAT;

/**
 * Stand-in for TornadoVM's FloatArray over libsoftbox_b200: the host copy is an off-heap
 * segment (what get/set touch, as before), the device copy a library allocation (what the
 * System downcalls receive). The copies are kept coherent lazily: get/set pull a newer
 * device copy first; a downcall uploads a newer host copy first.
 */
public final class FloatArray implements DeviceArray {
    private final int size;
    private final MemorySegment host;
    private MemorySegment dev;
    private boolean hostNewer = true;     // nothing on the device yet
    private boolean deviceNewer = false;

    public FloatArray(int numElements) {
        size = numElements;
        host = Arena.global().allocate(4L * Math.max(1, numElements), 16);
    }

    public static FloatArray fromElements(float... values) {
        FloatArray a = new FloatArray(values.length);
        for (int i = 0; i < values.length; i++) a.set(i, values[i]);
        return a;
    }

    public int getSize() { return size; }

    public float get(int i) {
        if (deviceNewer) syncToHost();
        return host.getAtIndex(JAVA_FLOAT, i);
    }

    public void set(int i, float v) {
        if (deviceNewer) syncToHost();
        host.setAtIndex(JAVA_FLOAT, i, v);
        hostNewer = true;
    }

    public void init(float v) {
        if (deviceNewer) syncToHost();
        for (int i = 0; i < size; i++) host.setAtIndex(JAVA_FLOAT, i, v);
        hostNewer = true;
    }

    public void clear() { init((float) 0); }

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
