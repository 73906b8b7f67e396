class HaloUpdater:
    pass
