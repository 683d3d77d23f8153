package softbox_b200.shim;

import java.lang.foreign.MemorySegment;

/**
 * An array with a host segment and a device allocation. Which copy is current is tracked:
 * a host write makes the host copy newer, a downcall that received the array makes the
 * device copy newer; reading the other side first copies the newer one over.
 */
public interface DeviceArray {
    /** The device pointer (allocated on first use, current contents uploaded). */
    MemorySegment dev();

    /** Uploads the host copy if it is newer than the device copy. */
    void syncToDevice();

    /** Records that a kernel may have written the device copy. */
    void markDeviceNewer();

    /** Downloads the device copy if it is newer than the host copy. */
    void syncToHost();

    /** Forces an upload at the next device use (EVERY_EXECUTION transfers). */
    void markHostNewer();
}
