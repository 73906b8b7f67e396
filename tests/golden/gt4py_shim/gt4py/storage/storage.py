import numpy as np


class Storage(np.ndarray):
    default_origin = None
    mask = None

    def __array_finalize__(self, obj):
        if obj is None:
            return
        self.default_origin = getattr(obj, "default_origin", None)
        self.mask = getattr(obj, "mask", None)

    def synchronize(self):
        pass

    def host_to_device(self, force=False):
        pass

    def device_to_host(self, force=False):
        pass

    def _set_device_modified(self):
        pass

    def _set_host_modified(self):
        pass
