package softbox_b200.shim;

/** A failing status of libsoftbox_b200 (SBX_EINVAL -1 ... SBX_ESTATE -7), with its message. */
public final class SbxException extends RuntimeException {
    public final int status;

    public SbxException(int status, String message) {
        super("softbox_b200 status " + status + ": " + message);
        this.status = status;
    }
}
