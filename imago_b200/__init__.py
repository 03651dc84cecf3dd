"""B200 integral setup for Imago: overlap, kinetic, nuclear and electronic
potential integrals over contracted GTOs, lattice-summed and Bloch-phased
onto every k-point, on sm_100a through the C ABI in include/imago_intg.h."""

from .system import AtomType, ImagoSystem, PotType, kpoint_mesh, pot_alphas  # noqa: F401
