"""Test-only stand-in for ``chex``: ``chex.dataclass`` as a stdlib dataclass
with a ``replace`` method (the only chex features the reference uses)."""
import dataclasses


def dataclass(cls=None, *, frozen=False, **kwargs):
    def wrap(c):
        d = dataclasses.dataclass(frozen=frozen, eq=False)(c)

        def replace(self, **changes):
            return dataclasses.replace(self, **changes)

        d.replace = replace
        return d

    return wrap if cls is None else wrap(cls)
