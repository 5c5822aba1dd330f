"""Import-only stand-in for matplotlib, used when importing the phasefield5d
reference to generate golden vectors (its solver package imports matplotlib
at module top for plotting, which the generator never calls)."""


def use(*args, **kwargs):
    return None
