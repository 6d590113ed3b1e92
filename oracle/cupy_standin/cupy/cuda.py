"""``cupy.cuda`` stand-in: stream synchronisation is a no-op on the CPU (test infrastructure only)."""


class _NullStream:
    def synchronize(self):
        return None


class Stream:
    null = _NullStream()


class runtime:
    @staticmethod
    def getDeviceCount():
        return 0
