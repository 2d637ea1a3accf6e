"""Inert pyplot stand-in (no plotting happens in fixture generation)."""


def __getattr__(name):
    def _noop(*args, **kwargs):
        return None

    return _noop
