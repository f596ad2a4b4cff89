"""Exception names the reference imports from gpubackendtools (cutils/__init__.py:10)."""


class BackendUnavailableException(Exception):
    pass


class MissingDependencies(Exception):
    def __init__(self, msg="", pip_deps=None, conda_deps=None):
        super().__init__(msg)
        self.pip_deps = pip_deps
        self.conda_deps = conda_deps


class CuPyException(Exception):
    pass
