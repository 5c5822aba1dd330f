"""Import-only stand-in for the formatter classes the reference imports."""


class FormatStrFormatter:
    def __init__(self, *args, **kwargs):
        pass


class ScalarFormatter:
    def __init__(self, *args, **kwargs):
        pass


class FuncFormatter:
    def __init__(self, *args, **kwargs):
        pass
