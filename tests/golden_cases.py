"""Cases behind the committed golden fixtures in tests/golden/ (made by
tests/golden/make_golden.py from the reference's own CPU build)."""

import parity_util as pu

CASES = {
    # name: (case factory, scheme)
    "cg_halfspace": (lambda: pu.small_halfspace(steps=40, NX=24, NY=22, NZ=18, nPML=5), "CGFDM"),
    "cg_hill_fault": (lambda: pu.multi_fault(steps=40, NX=26, NY=24, NZ=20, nPML=5), "CGFDM"),
    "cg_ricker": (lambda: pu.ricker_point(steps=40, NX=24, NY=24, NZ=18, nPML=5), "CGFDM"),
}


def hill_fault():
    c = pu.multi_fault(steps=40, NX=26, NY=24, NZ=20, nPML=5, courant=0.45)
    c.gauss_hill = 1
    return c


CASES["cg_hill_fault"] = (hill_fault, "CGFDM")


def sc_hill():
    c = pu.small_hill(steps=24, NX=24, NY=22, NZ=18, nPML=5)
    return c


CASES["sc_hill"] = (sc_hill, "SCFDM")
