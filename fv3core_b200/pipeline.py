"""Host-to-host streaming of states through one AcousticDynamics.

A caller whose states live in host memory (a driver that keeps the model
state on the CPU between dynamics steps, or a batch of independent states)
pays for the host-to-device copy of each state's inputs and the copy of its
results back.  ``StreamedAcoustics`` hides most of that cost: it keeps two
device copies of the state and runs three CUDA streams, so that while one
state is being advanced, the next state's inputs are being copied in and
the previous state's results are being copied out (H2D and D2H use the two
copy engines).  Every state still makes the full round trip; only the
waiting is overlapped.  The acoustic calls themselves stay in order on one
stream, because they share the context's workspace.
"""
import torch


class StreamedAcoustics:
    """``dynamics``: an AcousticDynamics.  ``states``: two device states (the
    namespaces ``AcousticDynamics.__call__`` takes) with the same scalars.
    ``inputs`` / ``outputs``: the field names copied in before and out after
    each call."""

    def __init__(self, dynamics, states, inputs, outputs):
        if len(states) != 2:
            raise ValueError("StreamedAcoustics needs exactly two device states")
        self.dynamics = dynamics
        self.states = states
        self.inputs = tuple(inputs)
        self.outputs = tuple(outputs)
        self.h2d = torch.cuda.Stream()
        self.compute = torch.cuda.Stream()
        self.d2h = torch.cuda.Stream()
        self._drained = [None, None]

    def run(self, batches):
        """Advance each (host_inputs, host_outputs) pair in order: copy the
        inputs (dicts of pinned host tensors by field name) into a device
        state, make one AcousticDynamics call, copy the outputs back.
        Returns when every copy has been enqueued; synchronise (or wait on
        ``self.d2h``) before reading the host outputs."""
        for n, (host_in, host_out) in enumerate(batches):
            slot = n % 2
            state = self.states[slot]
            # the slot's previous results must be out before new inputs go in
            if self._drained[slot] is not None:
                self.h2d.wait_event(self._drained[slot])
            with torch.cuda.stream(self.h2d):
                for k in self.inputs:
                    getattr(state, k).copy_(host_in[k], non_blocking=True)
                loaded = torch.cuda.Event()
                loaded.record(self.h2d)
            self.compute.wait_event(loaded)
            with torch.cuda.stream(self.compute):
                self.dynamics(state)
                computed = torch.cuda.Event()
                computed.record(self.compute)
            self.d2h.wait_event(computed)
            with torch.cuda.stream(self.d2h):
                for k in self.outputs:
                    host_out[k].copy_(getattr(state, k), non_blocking=True)
                drained = torch.cuda.Event()
                drained.record(self.d2h)
            self._drained[slot] = drained

    def synchronize(self):
        for s in (self.h2d, self.compute, self.d2h):
            s.synchronize()
