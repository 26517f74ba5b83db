"""get_ns_mesh / k-vector generation, delegating to the oracle restatement."""
from oracle.torchpme_shim import generate_kvectors, get_ns_mesh  # noqa: F401


def _generate_kvectors(cell, ns, for_ewald):
    return generate_kvectors(cell, ns, for_ewald)


def generate_kvectors_for_ewald(ns, cell):
    return generate_kvectors(cell, ns, True)
