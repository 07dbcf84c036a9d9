"""hp geometric multigrid (placeholder until the hierarchy builder lands)."""


class GeometricMultigridPreconditioner:
    def __init__(self, **kwargs):
        self.options = kwargs


def build_multigrid(plan, options):
    raise NotImplementedError("multigrid hierarchy")
