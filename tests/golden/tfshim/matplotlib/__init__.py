"""Inert matplotlib stand-in so the reference package imports without it
(plotting is never called by the fixture generator)."""


def use(*args, **kwargs):
    pass


def __getattr__(name):
    raise AttributeError(name)
