"""CPU restatement of the Kubo.PDOS start-vector selections -- TEST INFRASTRUCTURE ONLY.

Only tests/ import this module; it checks the library's gbn_pdos_atoms / gbn_pdos_sets and the
start vectors of gbn_lanczos_sites / gbn_lanczos_sets.  It follows the reference's loops literally,
whole-array coordinate conversions included:
  selections          lanczosKuboCode/Src/calc.F90:214-541 (CalcKubo, the Kubo.PDOS branch)
  conversions         atoms.F90:1768-1830 (AtomsSetCart, AtomsSetFrac)
  start vectors       kubo.F90:87-274 (KuboInitWFPDOS, KuboInitWFLayerDOS, KuboInitWFLayerAndSpeciesDOS)
Positions are (n, 3) Cartesian arrays; ucell is the flat 9-vector of the library (vector b at [3b:3b+3]).
"""

import numpy as np

LAYER, LAYER_SPECIES, DIST, MOIRE_SC1, SUPERMOIRE, SUPERMOIRE2, SUPERMOIRE3, ATOM_LIST, BY_NUMBER, PNP = range(1, 11)


class Atoms:
    """The atoms module's Rat with its frac flag."""

    def __init__(self, rat, ucell):
        self.r = np.array(rat, np.float64).reshape(-1, 3).copy()
        self.u = np.asarray(ucell, np.float64)
        self.frac = False

    def set_frac(self):   # atoms.F90:1796-1830
        if self.frac:
            return
        u11, u21, u12, u22, u33 = self.u[0], self.u[1], self.u[3], self.u[4], self.u[8]
        r = self.r
        assert u11 != 0.0
        r[:, 1] = u11 * (r[:, 1] - r[:, 0] * u21 / u11) / (u22 * u11 - u12 * u21)
        r[:, 0] = (r[:, 0] - r[:, 1] * u12) / u11
        r[:, 2] = r[:, 2] / u33
        self.frac = True

    def set_cart(self):   # atoms.F90:1768-1794
        if not self.frac:
            return
        f = self.r.copy()
        for k in range(3):
            self.r[:, k] = f[:, 0] * self.u[k] + f[:, 1] * self.u[3 + k] + f[:, 2] * self.u[6 + k]
        self.frac = False


def select_atoms(mode, rat, species, layer, ucell, xmin=0.0, xmax=5.0, ymin=0.0, ymax=5.0, min_value=0,
                 super_cell=1, cell_size=50, supermoire_length=135.0, aG=2.46, ignore_layers_1_4=False,
                 atom_list=(1, 2, 3, 4, 5, 6), atom_number=1, pnp_delta=10.0):
    """[(atom (1-based), coords line values)] in the order CalcKubo visits them."""
    at = Atoms(rat, ucell)
    n = len(at.r)
    out = []
    if mode == DIST:   # calc.F90:362-380
        at.set_cart()
        for i in range(1, n + 1):
            x, y = at.r[i - 1, 0], at.r[i - 1, 1]
            if x > xmin and x < xmax and y > ymin and y < ymax and i >= min_value:
                out.append((i, tuple(at.r[i - 1])))
    elif mode == MOIRE_SC1:   # calc.F90:381-402
        for i in range(1, n + 1):
            at.set_frac()
            if at.r[i - 1, 0] < 1.0 / super_cell and at.r[i - 1, 1] < 1.0 / super_cell and i >= min_value:
                if ignore_layers_1_4 and layer[i - 1] in (1, 4):
                    continue
                at.set_cart()
                out.append((i, (at.r[i - 1, 0], at.r[i - 1, 1], int(species[i - 1]), int(layer[i - 1]))))
    elif mode in (SUPERMOIRE, SUPERMOIRE2, SUPERMOIRE3):   # calc.F90:403-467
        length = supermoire_length / aG
        t = [k / super_cell / cell_size * length for k in (1.0, 2.0, 3.0)]
        for i in range(1, n + 1):
            at.set_frac()
            fx, fy = at.r[i - 1, 0], at.r[i - 1, 1]
            if mode == SUPERMOIRE:
                sel = fx < t[0] and (fy < t[0] and species[i - 1] == 1 and i >= min_value)
            elif mode == SUPERMOIRE2:
                sel = fx >= t[0] and (fy >= t[0] and fx < t[1] and fy < t[1] and species[i - 1] == 1 and i >= min_value)
            else:
                sel = fx >= t[1] and (fy >= t[1] and fx < t[2] and fy < t[2] and species[i - 1] == 1 and i >= min_value)
            if sel:
                at.set_cart()
                out.append((i, tuple(at.r[i - 1])))
    elif mode == ATOM_LIST:   # calc.F90:471-487
        for i in atom_list:
            out.append((i, tuple(at.r[i - 1])))
    elif mode == BY_NUMBER:   # calc.F90:489-493
        out.append((atom_number, tuple(at.r[atom_number - 1])))
    elif mode == PNP:   # calc.F90:494-541
        at.set_cart()
        acc = aG / np.sqrt(3.0)
        limit1 = (cell_size * super_cell * aG) * 1.0 / 4.0
        f1 = f2 = False
        for i in range(1, n + 1):
            x = at.r[i - 1, 0]
            if x > limit1 and x < limit1 + acc and not f1:
                f1 = True
                out.append((i, tuple(at.r[i - 1])))
            if x > limit1 + pnp_delta * 2.0 and x < limit1 + pnp_delta * 2.0 + acc and not f2:
                f2 = True
                out.append((i, tuple(at.r[i - 1])))
    else:
        raise ValueError(mode)
    return out


def layer_sets(mode, species, layer, number_of_layers=2, super_cell=1, stack=0, n_bn1=5832, n_bn2=5832, n_c=6050):
    """[(layer, species or 0, assumed count, member mask)] of Kubo.PDOSLayer / PDOSLayerAndSpecies
    (calc.F90:300-361); stack 1 = Stack.EncapsulatedFourLayers, 2 = Stack.T3BG."""
    n = len(layer)
    sets = []
    if mode == LAYER:
        for i in range(1, number_of_layers + 1):
            if i in (1, 2, 3, 4) and stack == 2:
                m = n_c * super_cell * super_cell
            elif i in (5, 6) and stack == 2:
                m = n_c * super_cell * super_cell
            elif i == 1 and stack == 1:
                m = n_bn1 * super_cell * super_cell
            elif i == 4 and stack == 1:
                m = n_bn2 * super_cell * super_cell
            elif i in (2, 3) and stack == 1:
                m = n_c * super_cell * super_cell
            else:
                m = n // number_of_layers
            sets.append((i, 0, m, np.asarray(layer) == i))
    else:
        max_species = max(1, int(np.max(species)))
        for i in range(1, number_of_layers + 1):
            for ii in range(1, max_species + 1):
                mask = (np.asarray(layer) == i) & (np.asarray(species) == ii)
                m = int(mask.sum())
                if m == 0:
                    continue
                sets.append((i, ii, m, mask))
    return sets


def layer_start_vector(mask, assumed, draws):
    """KuboInitWFLayerDOS (kubo.F90:140-212): phases on the set's atoms from a reseeded stream, scaled by
    1/sqrt(assumed) and normalised when the norm then differs from 1 by more than 1e-6."""
    n = len(mask)
    psi = np.zeros(n, np.complex128)
    k = 0
    for i in range(n):
        if mask[i]:
            psi[i] = np.exp(2.0 * np.pi * 1j * draws[k]) / np.sqrt(float(assumed))
            k += 1
    cnum = float(np.sum((psi * np.conj(psi)).real))
    if cnum > 0.0 and abs(cnum - 1.0) > 1.0e-6:
        psi = psi / np.sqrt(cnum)
    return psi


def site_start_vector(n, atom):
    """KuboInitWFPDOS (kubo.F90:87-138): 1 on the atom, 0 elsewhere."""
    psi = np.zeros(n, np.complex128)
    psi[atom - 1] = 1.0
    return psi
