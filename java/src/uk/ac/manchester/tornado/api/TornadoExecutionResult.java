package uk.ac.manchester.tornado.api;

import softbox_b200.shim.DeviceArray;

/** Stand-in: transferToHost pulls the device copies of the given arrays (UNDER_DEMAND). */
public final class TornadoExecutionResult {
    public TornadoExecutionResult transferToHost(Object... arrays) {
        for (Object o : arrays) if (o instanceof DeviceArray d) d.syncToHost();
        return this;
    }
}
