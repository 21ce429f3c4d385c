"""Host containers mirroring the reference's aero pytrees.

``GridDiscretisation`` (aero/data_structures.py:29-40), ``ArrayList`` and
``ArrayListShape`` (algebra/array_utils.py:139-322), ``AeroStates``
(aero/gradients/data_structures.py:113-193) and ``AeroCase``
(aero/data_structures.py:43-615) with the same field names and per-surface layouts: a
snapshot holds ``(m+1, n+1, 3)`` lattices and ``(m, n)`` circulations per surface; a
batched case adds a leading time axis.  ``project_forcing_to_beam`` (aero/utils.py:666-697)
is the O(M N) host reduction the reference's fluid-structure loop applies to a solved slot.
"""
from __future__ import annotations

from collections import OrderedDict
from dataclasses import dataclass

import numpy as np


@dataclass
class GridDiscretisation:
    """Chordwise, spanwise and wake panel counts of one surface."""

    m: int
    n: int
    m_star: int


class ArrayListShape:
    """Shapes of the arrays of an ArrayList (algebra/array_utils.py:293-322)."""

    def __init__(self, shapes):
        self.shapes = [tuple(s) for s in shapes]
        self.n_arrays = len(self.shapes)
        self.sizes = [int(np.prod(s, dtype=np.int64)) for s in self.shapes]

    def __iter__(self):
        return iter(self.shapes)

    def __len__(self):
        return self.n_arrays

    def __getitem__(self, i):
        return self.shapes[i]

    def __eq__(self, other):
        return isinstance(other, ArrayListShape) and self.shapes == other.shapes

    def __repr__(self):
        return f"ArrayListShape(n_arrays={self.n_arrays}), shapes={self.shapes}"

    def total_size(self) -> int:
        return sum(self.sizes)


class ArrayList(list):
    """A list of per-surface arrays with elementwise arithmetic, as the reference's
    ``ArrayList`` (algebra/array_utils.py:139-290): ``a + b`` adds surface by surface,
    ``ravel`` concatenates the flattened arrays in surface order."""

    def index_all(self, *idx):
        return ArrayList([a[idx] for a in self])

    def copy(self):
        return ArrayList([np.array(a, copy=True) for a in self])

    # elementwise arithmetic (the list operators would concatenate or repeat)
    def __add__(self, other):
        return ArrayList([a + b for a, b in zip(self, other, strict=True)])

    def __iadd__(self, other):
        for i, b in enumerate(other):
            self[i] = self[i] + b
        return self

    def __sub__(self, other):
        return ArrayList([a - b for a, b in zip(self, other, strict=True)])

    def __isub__(self, other):
        for i, b in enumerate(other):
            self[i] = self[i] - b
        return self

    def __neg__(self):
        return ArrayList([-a for a in self])

    def __mul__(self, val):
        return ArrayList([a * val for a in self])

    def __rmul__(self, val):
        return self.__mul__(val)

    def __imul__(self, val):
        for i in range(len(self)):
            self[i] = self[i] * val
        return self

    def __truediv__(self, val):
        return ArrayList([a / val for a in self])

    def __rtruediv__(self, val):
        return ArrayList([val / a for a in self])

    def __matmul__(self, other):
        return ArrayList([a @ b for a, b in zip(self, other, strict=True)])

    def to_list(self):
        return list(self)

    def at(self, idx: int):
        return self[idx]

    def combine(self, *others):
        out = ArrayList(self)
        for o in others:
            out.extend(o)
        return out

    def ravel(self) -> np.ndarray:
        """The arrays flattened and concatenated in surface order."""
        if len(self) == 0:
            return np.zeros(0)
        return np.concatenate([np.ravel(a) for a in self])

    @classmethod
    def from_vector(cls, vect, shapes: ArrayListShape) -> "ArrayList":
        """Inverse of ``ravel`` for the given shapes (algebra/array_utils.py:212-235)."""
        vect = np.asarray(vect)
        if vect.size != sum(shapes.sizes):
            raise ValueError(
                f"Input vector must have the same number of elements as shapes. Vector has "
                f"{vect.size} elements, but shape requires {sum(shapes.sizes)}.")
        out, i = [], 0
        for shape, size in zip(shapes.shapes, shapes.sizes):
            out.append(vect[i:i + size].reshape(shape))
            i += size
        return cls(out)

    @staticmethod
    def einsum(subscript: str, *operands) -> "ArrayList":
        n = len(operands[0])
        if any(len(op) != n for op in operands):
            raise ValueError("All ArrayLists must have the same length.")
        return ArrayList([np.einsum(subscript, *(op[i] for op in operands)) for i in range(n)])

    @staticmethod
    def zeros_like(arr) -> "ArrayList":
        return ArrayList([np.zeros_like(a) for a in arr])

    @property
    def shape(self) -> ArrayListShape:
        return ArrayListShape([np.shape(a) for a in self])

    @property
    def size(self) -> int:
        return int(sum(np.size(a) for a in self))


class AeroStates:
    """The aerodynamic states of one time step (aero/gradients/data_structures.py:113-193):
    bound and wake circulations, the bound circulation rate and the wake lattice, raveled in
    that order."""

    def __init__(self, gamma_b, gamma_w, gamma_b_dot, zeta_w):
        self.gamma_b = ArrayList(gamma_b)
        self.gamma_w = ArrayList(gamma_w)
        self.gamma_b_dot = ArrayList(gamma_b_dot)
        self.zeta_w = ArrayList(zeta_w)

    def shapes(self) -> OrderedDict:
        return OrderedDict(gamma_b=self.gamma_b.shape, gamma_w=self.gamma_w.shape,
                           gamma_b_dot=self.gamma_b_dot.shape, zeta_w=self.zeta_w.shape)

    @staticmethod
    def from_vector(vect, shapes: OrderedDict) -> "AeroStates":
        """Inverse of ``ravel`` (``vect_to_arrs``, algebra/array_utils.py:374-403)."""
        vect = np.asarray(vect)
        out, i = {}, 0
        for name, shape in shapes.items():
            n = shape.total_size()
            out[name] = ArrayList.from_vector(vect[i:i + n], shape)
            i += n
        if i != vect.size:
            raise ValueError(f"state vector has {vect.size} entries, the shapes need {i}")
        return AeroStates(**out)

    def ravel(self) -> np.ndarray:
        return np.concatenate([self.gamma_b.ravel(), self.gamma_w.ravel(), self.gamma_b_dot.ravel(),
                               self.zeta_w.ravel()])

    @property
    def n_states(self) -> int:
        return self.gamma_b.size + self.gamma_w.size + self.gamma_b_dot.size + self.zeta_w.size


def project_forcing_to_beam(f_total, rmat, dof_mapping, x0_aero) -> np.ndarray:
    """Vertex forces summed onto the beam nodes, ``(n_nodes, 6)`` in the global frame
    (aero/utils.py:666-697).

    For each surface and spanwise vertex column j mapped to node ``dof_mapping[j]``: the
    force is the column's sum of vertex forces, the moment the column's sum of
    ``(R_node x0) x f`` with ``x0`` the vertex's reference coordinates.  As in the
    reference, a node that several surfaces map to keeps the last surface's values.
    """
    rmat = np.asarray(rmat, dtype=np.float64)
    out = np.zeros((rmat.shape[0], 6))
    for f, x0, dof in zip(f_total, x0_aero, dof_mapping):
        f = np.asarray(f, dtype=np.float64)
        dof = np.asarray(dof)
        r_x0 = np.einsum("jab,ijb->ija", rmat[dof], np.asarray(x0, dtype=np.float64))
        out[dof, :3] = f.sum(axis=0)
        out[dof, 3:] = np.cross(r_x0, f).sum(axis=0)
    return out


_FIELDS = ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
           "f_unsteady", "alpha")


class AeroCase:
    """UVLM solution over one (snapshot) or many (batched) time steps.

    Fields as the reference: ``zeta_b, zeta_b_dot, zeta_w, c, nc, gamma_b, gamma_b_dot,
    gamma_w, f_steady, f_unsteady, alpha`` (ArrayLists), ``t`` and ``i_ts``.  ``force_total``
    (per slot, sum over every vertex of ``f_steady + f_unsteady``) is an addition.
    """

    def __init__(self, zeta_b, zeta_b_dot, zeta_w, c, n, gamma_b, gamma_b_dot, gamma_w, f_steady, f_unsteady, alpha,
                 t, i_ts, force_total=None, **meta):
        self.zeta_b = ArrayList(zeta_b)
        self.zeta_b_dot = ArrayList(zeta_b_dot)
        self.zeta_w = ArrayList(zeta_w)
        self.c = ArrayList(c)
        self.nc = ArrayList(n)
        self.gamma_b = ArrayList(gamma_b)
        self.gamma_b_dot = ArrayList(gamma_b_dot)
        self.gamma_w = ArrayList(gamma_w)
        self.f_steady = ArrayList(f_steady)
        self.f_unsteady = ArrayList(f_unsteady)
        self.alpha = ArrayList(alpha)
        self.t = np.asarray(t, dtype=np.float64)
        self.i_ts = i_ts
        self.force_total = None if force_total is None else np.asarray(force_total)
        self.meta = meta

    @property
    def is_batched(self) -> bool:
        return self.gamma_b[0].ndim == 3  # aero/data_structures.py:161-164

    @property
    def n_tstep(self) -> int:
        if not self.is_batched:
            raise TypeError("n_tstep only defined for a batched AeroCase")
        return self.gamma_b[0].shape[0]

    def _fields(self):
        return {k: getattr(self, k) for k in _FIELDS}

    def __getitem__(self, idx: int) -> "AeroCase":
        """Snapshot at time index ``idx`` (aero/data_structures.py:533-568)."""
        if not self.is_batched:
            raise TypeError("__getitem__ only supported for batched AeroCase")
        f = {k: [a[idx] for a in v] for k, v in self._fields().items()}
        f["n"] = f.pop("nc")
        ft = None if self.force_total is None else self.force_total[idx]
        return AeroCase(**f, t=self.t[idx], i_ts=idx, force_total=ft, **self.meta)

    def to_dynamic(self, i_ts: int, n_tstep: int) -> "AeroCase":
        """Expand a snapshot into ``n_tstep`` zero-filled slots with the snapshot at
        ``i_ts`` (aero/data_structures.py:570-610)."""
        if self.is_batched:
            raise TypeError("to_dynamic only supported for snapshot AeroCase")
        f = {}
        for k, v in self._fields().items():
            out = []
            for a in v:
                z = np.zeros((n_tstep,) + np.shape(a))
                z[i_ts] = a
                out.append(z)
            f[k] = out
        f["n"] = f.pop("nc")
        t = np.zeros(n_tstep)
        t[i_ts] = self.t
        ft = None
        if self.force_total is not None:
            ft = np.zeros((n_tstep, 3))
            ft[i_ts] = self.force_total
        return AeroCase(**f, t=t, i_ts=np.arange(n_tstep), force_total=ft, **self.meta)

    def set_arraylist_at_ts(self, attr: str, values, i_ts: int) -> None:
        if not self.is_batched:
            raise TypeError("set_arraylist_at_ts only supported for batched AeroCase")
        arr = getattr(self, attr)
        for i, val in enumerate(values):
            arr[i][i_ts] = val

    @classmethod
    def initialise(cls, initial_snapshot: "AeroCase", n_tstep: int) -> "AeroCase":
        """A batched case with ``initial_snapshot`` at slot 0 (aero/data_structures.py:612-615)."""
        return initial_snapshot.to_dynamic(i_ts=0, n_tstep=n_tstep)

    @property
    def n_surf(self) -> int:
        return len(self.gamma_b)

    @property
    def dof_mapping(self):
        """Vertex column -> beam node, per surface (set by the UVLM that made the case)."""
        return self.meta.get("dof_mapping")

    @property
    def flowfield(self):
        return self.meta.get("flowfield")

    def _slot(self, field, i_ts):
        arr = getattr(self, field)
        if self.is_batched:
            if i_ts is None:
                raise ValueError("i_ts must be provided for batched AeroCase")
            return arr.index_all(i_ts, ...)
        return ArrayList(arr)

    def get_states(self, i_ts=None) -> AeroStates:
        """The AeroStates of slot ``i_ts`` (aero/data_structures.py:240-266)."""
        return AeroStates(gamma_b=self._slot("gamma_b", i_ts), gamma_w=self._slot("gamma_w", i_ts),
                          gamma_b_dot=self._slot("gamma_b_dot", i_ts), zeta_w=self._slot("zeta_w", i_ts))

    def gamma_full(self, i_ts=None) -> ArrayList:
        """Bound then wake circulations, ``(2 n_surf,)`` arrays (aero/data_structures.py:268-282)."""
        return self._slot("gamma_b", i_ts).combine(self._slot("gamma_w", i_ts))

    def zeta_full(self, i_ts=None) -> ArrayList:
        """Bound then wake lattices, ``(2 n_surf,)`` arrays (aero/data_structures.py:284-298)."""
        return self._slot("zeta_b", i_ts).combine(self._slot("zeta_w", i_ts))

    def __setitem__(self, i_ts: int, snapshot: "AeroCase") -> None:
        """Write a snapshot into slot ``i_ts`` (aero/data_structures.py:357-412)."""
        if not self.is_batched:
            raise TypeError("__setitem__ only supported for batched AeroCase")
        if snapshot.is_batched:
            raise TypeError("snapshot AeroCase must not be batched")
        self.t[i_ts] = snapshot.t
        for k in _FIELDS:
            if k in ("c", "nc"):
                continue  # the reference leaves the geometry caches alone
            self.set_arraylist_at_ts(k, getattr(snapshot, k), i_ts)
        if self.force_total is not None and snapshot.force_total is not None:
            self.force_total[i_ts] = snapshot.force_total

    def project_forcing_to_beam(self, i_ts, rmat, x0_aero, include_unsteady: bool) -> np.ndarray:
        """Slot ``i_ts``'s vertex forces onto the beam nodes, ``(n_nodes, 6)`` (forces, then
        moments of ``R x0`` about each node), the call the reference's fluid-structure loop
        makes after every ``case_solve`` (aero/data_structures.py:464-492,
        structure/beam.py:2656-2674)."""
        if self.dof_mapping is None:
            raise ValueError("this AeroCase carries no dof_mapping (build it through UVLM)")
        f = self._slot("f_steady", i_ts)
        if include_unsteady:
            f = f + self._slot("f_unsteady", i_ts)
        return project_forcing_to_beam(f, rmat, self.dof_mapping, x0_aero)

    def _t_at(self, i_ts):
        if self.is_batched:
            if i_ts is None:
                raise ValueError("i_ts required for batched AeroCase")
            return float(self.t[i_ts])
        return float(self.t)

    def get_v_background(self, x_target, i_ts=None):
        """Background flow at points (aero/data_structures.py:500-509): an array of points,
        or an ArrayList of per-surface point arrays."""
        t = self._t_at(i_ts)
        if isinstance(x_target, ArrayList):
            return ArrayList([self.flowfield(np.asarray(x, float), t) for x in x_target])
        return self.flowfield(np.asarray(x_target, float), t)

    def get_v_ind(self, x_target, i_ts=None):
        """Induced velocity of every bound and wake lattice of slot ``i_ts`` at points
        (aero/data_structures.py:511-524), summed on the device by ``fj_vind`` with the
        kernel, mirror plane and precision of the UVLM that made the case."""
        solver = self.meta.get("induced")
        if solver is None:
            raise ValueError("this AeroCase carries no induced-velocity settings (build it through UVLM)")
        zetas, gammas = self.zeta_full(i_ts), self.gamma_full(i_ts)
        if isinstance(x_target, ArrayList):
            pts = [np.asarray(x, float) for x in x_target]
            flat = np.concatenate([p.reshape(-1, 3) for p in pts])
            v = solver(flat, zetas, gammas)
            out, o = ArrayList(), 0
            for p in pts:
                n = p.size // 3
                out.append(v[o:o + n].reshape(p.shape))
                o += n
            return out
        x = np.asarray(x_target, float)
        return solver(x.reshape(-1, 3), zetas, gammas).reshape(x.shape)

    def get_v_tot(self, x_target, i_ts=None):
        """Induced plus background velocity (aero/data_structures.py:526-531)."""
        return self.get_v_ind(x_target, i_ts) + self.get_v_background(x_target, i_ts)
