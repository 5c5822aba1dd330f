"""Import-only stand-in: every attribute is a no-op callable."""


def __getattr__(name):
    def _noop(*args, **kwargs):
        return None
    return _noop
