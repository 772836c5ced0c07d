"""Bonded interaction objects mirroring ``espressomd.interactions``
(script_interface/interactions/BondedInteraction.hpp): ``FeneBond`` and
``HarmonicBond``.  Register them with ``system.bonded_inter.add(bond)`` and
attach them with ``particle.add_bond((bond, partner))``; forces, energies
and virials come from libp3mx.so (p3mx_set_bonds, p3mx_bond_observables).
"""
from . import _lib


class BondedInteraction:
    _kind = 0

    def params(self):
        raise NotImplementedError

    def c_params(self):
        k, r0, r_max = self.params()
        return _lib.BondParams(self._kind, k, r0, r_max)


class FeneBond(BondedInteraction):
    """FENE bond (bonded_interactions/fene.hpp:37-105):
    F(r) = -k (r - r_0) / (1 - ((r - r_0) / d_r_max)^2) along the bond,
    E(r) = -k d_r_max^2 / 2 ln(1 - ((r - r_0) / d_r_max)^2); broken for
    r - r_0 >= d_r_max."""
    _kind = _lib.P3MX_BOND_FENE

    def __init__(self, k, d_r_max, r_0=0.0):
        if d_r_max <= 0:
            raise ValueError("FENE parameter 'd_r_max' has to be > 0")
        self.k, self.d_r_max, self.r_0 = float(k), float(d_r_max), float(r_0)

    def params(self):
        return self.k, self.r_0, self.d_r_max

    def get_params(self):
        return dict(k=self.k, d_r_max=self.d_r_max, r_0=self.r_0)


class HarmonicBond(BondedInteraction):
    """Harmonic bond (bonded_interactions/harmonic.hpp:35-93):
    F(r) = -k (r - r_0), E(r) = k (r - r_0)^2 / 2; broken for r > r_cut when
    r_cut > 0."""
    _kind = _lib.P3MX_BOND_HARMONIC

    def __init__(self, k, r_0, r_cut=0.0):
        self.k, self.r_0, self.r_cut = float(k), float(r_0), float(r_cut)

    def params(self):
        return self.k, self.r_0, self.r_cut

    def get_params(self):
        return dict(k=self.k, r_0=self.r_0, r_cut=self.r_cut)


class BondedInteractions:
    """``system.bonded_inter``: the registered bond objects (bond ids in
    order of registration)."""

    def __init__(self, system):
        self._system = system
        self._bonds = []

    def add(self, bond):
        if not isinstance(bond, BondedInteraction):
            raise TypeError("only FeneBond and HarmonicBond are supported")
        if bond not in self._bonds:
            self._bonds.append(bond)
            self._system._bonds_changed()
        return self._bonds.index(bond)

    def clear(self):
        self._bonds = []
        self._system.part._bonds = []
        self._system._bonds_changed()

    def __getitem__(self, i):
        return self._bonds[i]

    def __len__(self):
        return len(self._bonds)

    def _id(self, bond):
        try:
            return self._bonds.index(bond)
        except ValueError:
            raise ValueError("the bond has to be added to system.bonded_inter first") from None
