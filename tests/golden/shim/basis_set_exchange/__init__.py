"""Test-only stand-in for ``basis_set_exchange``: serves BSE-schema dicts that
the fixture generator registers with ``register``; there is no basis database."""
import copy

_REGISTRY = {}


def register(name, data):
    _REGISTRY[name.lower()] = data


def get_basis(name, elements=None, uncontract_spdf=True, header=False):
    data = _REGISTRY[name.lower()]
    out = {"name": name, "elements": {}}
    for z in elements or []:
        key = str(int(z))
        if key in data["elements"]:
            out["elements"][key] = copy.deepcopy(data["elements"][key])
    return out


def get_all_basis_names():
    return sorted(_REGISTRY)
