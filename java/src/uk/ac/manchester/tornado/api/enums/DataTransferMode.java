package uk.ac.manchester.tornado.api.enums;

/** Stand-in for TornadoVM's transfer modes, mapped onto the shim's host/device coherence:
 *  FIRST_EXECUTION uploads once (at the first device use), EVERY_EXECUTION uploads at every
 *  execute(), UNDER_DEMAND downloads when transferToHost is called on the result. */
public enum DataTransferMode {
    FIRST_EXECUTION, EVERY_EXECUTION, UNDER_DEMAND
}
