"""Particles: device-resident macro-particle store with the reference API.

Mirrors ``particles.Particles`` (particles.pyx:14-197).  The reference keeps an
(N, 6) float64 AoS numpy array [x, y, vx, vy, vz, w]; here the particles live
on the GPU as FP32 structure-of-arrays with the position split into the cell
index and the in-cell offset (see include/oec.h).  Methods keep the
reference's names, arguments and meaning; getters return numpy copies
(the reference returns views -- a device store cannot hand out host views).

The position representation needs the grid, so a particle store binds to the
first Grid it is used with (``setParticleData`` before that keeps the rows on
the host until the grid is known).
"""
import numpy as np
import torch

from . import _lib
from . import device as D
from .constants import elementary_charge, m_e, m_p

CHUNK = 1024  # capacity granularity (kernel CTA chunk)


class Particles:
    def __init__(self, particleSpecies, particleType, capacity=0):
        if particleSpecies == "electrons":
            self.particleMass = m_e
            self.particleCharge = -elementary_charge
        elif particleSpecies == "protons":
            self.particleMass = m_p
            self.particleCharge = elementary_charge
        else:
            raise NotImplementedError("Not yet implemented.")
        if particleType != "variableWeight":
            raise NotImplementedError("Not yet implemented.")
        self.nCoords = 6
        self.dt = 0.0
        self.bConst = np.zeros(3)
        self._grid = None
        self._pending = np.empty((0, 6))
        self._cap = 0
        self._soa = None
        self._count = None
        self._status = None
        self._mask = None
        self._wscale = None
        self._min_capacity = int(capacity)
        self.chargeOnGrid = None       # device f64 [npExt]
        self._rho_fix = None           # device int64 [npExt]
        self.eAtParticles = None       # device f64 [N,2]
        self.bAtParticles = None       # device f64 [N,3]
        self._weights = None

    # ------------------------------------------------------------- storage
    def _alloc(self, cap):
        cap = D.round_up(max(cap, CHUNK), CHUNK)
        old, oldcap = self._soa, self._cap
        soa = {"cell": D.zeros(cap, torch.int32)}
        for k in ("ox", "oy", "vx", "vy", "vz", "w"):
            soa[k] = D.zeros(cap, torch.float32)
        if old is not None:
            n = min(oldcap, cap)
            for k in soa:
                soa[k][:n].copy_(old[k][:n])
        self._soa, self._cap = soa, cap
        if self._count is None:
            self._count = D.zeros(1, torch.int32)
            # row count of the reference's particle array (particles.pyx:109-116)
            self._array_len = D.zeros(1, torch.int32)
            self._status = D.zeros(_lib.STATUS_WORDS, torch.int32)
            self._wscale = D.zeros(1, torch.float64)
        mask = D.zeros(cap // 32, torch.int32)
        if self._mask is not None:  # keep the absorbed bits across a regrowth
            m = min(mask.shape[0], self._mask.shape[0])
            mask[:m].copy_(self._mask[:m])
        self._mask = mask

    def ensure_capacity(self, n):
        """Grow the device store (x1.5, like the reference's x1.1 regrowth) to hold n."""
        need = max(int(n), self._min_capacity)
        if need > self._cap or self._soa is None:
            self._alloc(max(need, int(self._cap * 1.5)))

    def c_particles(self):
        s = self._soa
        return _lib.Particles_t(s["cell"].data_ptr(), s["ox"].data_ptr(), s["oy"].data_ptr(),
                                s["vx"].data_ptr(), s["vy"].data_ptr(), s["vz"].data_ptr(),
                                s["w"].data_ptr(), self._count.data_ptr(), self._cap)

    def _bind(self, gridObj):
        if self._grid is None:
            self._grid = gridObj
            pend, self._pending = self._pending, None
            self._upload(pend)
        elif gridObj is not self._grid and gridObj.c_grid().nx != self._grid.c_grid().nx:
            raise ValueError("particle store is bound to a different grid")
        return self._grid

    def _upload(self, aos):
        aos = D.to_device(aos, torch.float64).reshape(-1, 6)
        n = aos.shape[0]
        self.ensure_capacity(n)
        p = self.c_particles()
        _lib.call("oec_particles_from_aos", self._grid.c_grid(), aos.data_ptr() if n else None, n, p, D.stream())
        self._array_len.fill_(n)

    def soa(self):
        return self._soa

    # --------------------------------------------------------------- API
    def setParticleData(self, particleData):
        """particles.pyx:126-140."""
        if isinstance(particleData, torch.Tensor):
            data = particleData
        else:
            data = np.ascontiguousarray(particleData, dtype=np.float64).reshape(-1, 6)
        if self._grid is None:
            self._pending = data if not isinstance(data, torch.Tensor) else data.cpu().numpy()
        else:
            self._upload(data)
        self.eAtParticles = None
        self.bAtParticles = None

    def getParticleData(self):
        """particles.pyx:142-143 (a host copy of the first count rows)."""
        if self._grid is None:
            return np.array(self._pending, copy=True)
        n = self.getMacroParticleCount()
        out = D.empty((max(n, 1), 6), torch.float64)
        _lib.call("oec_particles_to_aos", self._grid.c_grid(), self.c_particles(), out.data_ptr(), n, D.stream())
        return out[:n].cpu().numpy()

    def getParticleDataDevice(self):
        """Device (count, 6) float64 tensor of the particles (no host copy)."""
        n = self.getMacroParticleCount()
        out = D.empty((max(n, 1), 6), torch.float64)
        _lib.call("oec_particles_to_aos", self._grid.c_grid(), self.c_particles(), out.data_ptr(), n, D.stream())
        return out[:n]

    def getFullParticleData(self):
        return self.getParticleData()

    def getNCoords(self):
        return self.nCoords

    def getMacroParticleCount(self):
        if self._grid is None:
            return int(self._pending.shape[0])
        return int(self._count.item())

    def setMacroParticleCount(self, macroParticleCount):
        if self._grid is None:
            self._pending = self._pending[:int(macroParticleCount)]
        else:
            if int(macroParticleCount) > self._cap:
                raise ValueError("count exceeds capacity")
            self._count.fill_(int(macroParticleCount))

    def getParticleCharge(self):
        return self.particleCharge

    def getParticleMass(self):
        return self.particleMass

    def getDt(self):
        return self.dt

    def setBConst(self, bConst):
        """particles.pyx:123-124."""
        self.bConst = np.asarray(bConst, dtype=np.float64).reshape(3).copy()

    def getMeanWeight(self):
        """particles.pyx:39-47."""
        n = self.getMacroParticleCount()
        return float(self._soa["w"][:n].double().sum().item()) / n

    def sortByColumn(self, sortByColumn):
        """particles.pyx:49-50: reorder the particles by column 2..5
        (vx, vy, vz, w) of the reference layout, or 6 for the cell index
        (stable device radix sort; the reference uses a random-pivot quicksort,
        so only the order of equal keys can differ)."""
        col = int(sortByColumn)
        if col in (0, 1):
            col = 6  # x, y: the cell-major order is the position order used on the device
        if col not in (2, 3, 4, 5, 6):
            raise ValueError("column must be 0..5 (or 6 for cells)")
        tmp = self.c_scratch()
        if getattr(self, "_sort_work", None) is None or self._sort_work_cap != self._cap:
            self._sort_work = D.empty(int(_lib.lib().oec_sort_work_bytes(self._cap)), torch.uint8)
            self._sort_work_cap = self._cap
        _lib.call("oec_sort_particles", self.c_particles(), tmp, col, self._sort_work.data_ptr(), D.stream())
        self._soa, self._sort_tmp = self._sort_tmp, self._soa

    def c_scratch(self):
        """A second store of the same capacity: the sort's output (swapped in
        afterwards) and the staging area of the shifting add/remove rules."""
        if getattr(self, "_sort_tmp", None) is None or self._sort_tmp["cell"].shape[0] != self._cap:
            self._sort_tmp = {"cell": D.empty(self._cap, torch.int32)}
            for k in ("ox", "oy", "vx", "vy", "vz", "w"):
                self._sort_tmp[k] = D.empty(self._cap, torch.float32)
        t = self._sort_tmp
        return _lib.Particles_t(t["cell"].data_ptr(), t["ox"].data_ptr(), t["oy"].data_ptr(), t["vx"].data_ptr(),
                                t["vy"].data_ptr(), t["vz"].data_ptr(), t["w"].data_ptr(), self._count.data_ptr(),
                                self._cap)

    def calcGridWeights(self, gridObj):
        """particles.pyx:52-56 -> inCell and the four CIC weights (device)."""
        self._bind(gridObj)
        n = max(self._cap, CHUNK)
        if self._weights is None or self._weights[0].shape[0] < self._cap:
            self._weights = (D.empty(n, torch.int32),) + tuple(D.empty(n, torch.float64) for _ in range(4))
        inc, w00, w10, w01, w11 = self._weights
        _lib.call("oec_calc_grid_weights", gridObj.c_grid(), self.c_particles(), inc.data_ptr(), w00.data_ptr(),
                  w10.data_ptr(), w01.data_ptr(), w11.data_ptr(), D.stream())

    def _weight(self, k):
        n = self.getMacroParticleCount()
        return D.to_numpy(self._weights[k][:n])

    def getInCell(self):
        return self._weight(0).astype(np.uint32)

    def getWeightLowXLowY(self): return self._weight(1)
    def getWeightUpXLowY(self): return self._weight(2)
    def getWeightLowXUpY(self): return self._weight(3)
    def getWeightUpXUpY(self): return self._weight(4)

    def _deposit_buffers(self, gridObj):
        G = gridObj.getNpExt()
        if self._rho_fix is None or self._rho_fix.shape[0] != G:
            self._rho_fix = D.zeros(G, torch.int64)
            self.chargeOnGrid = D.zeros(G, torch.float64)

    def chargeToGrid(self, gridObj):
        """particles.pyx:70-77 as an int64 fixed-point deposit (order independent)."""
        self._bind(gridObj)
        self._deposit_buffers(gridObj)
        g, p, s = gridObj.c_grid(), self.c_particles(), D.stream()
        _lib.call("oec_deposit_scale", p, self._wscale.data_ptr(), s)
        _lib.call("oec_deposit", g, p, self._rho_fix.data_ptr(), self._wscale.data_ptr(), 1,
                  self._status.data_ptr(), s)
        _lib.call("oec_deposit_finalize", g, self._rho_fix.data_ptr(), self._wscale.data_ptr(),
                  self.particleCharge, self.chargeOnGrid.data_ptr(), s)

    def getChargeOnGrid(self):
        return D.to_numpy(self.chargeOnGrid)

    def getChargeOnGridDevice(self):
        return self.chargeOnGrid

    def getChargeOnGridFixed(self):
        """The int64 fixed-point deposit and its scale (charge = q * fix / wscale)."""
        return D.to_numpy(self._rho_fix), float(self._wscale.item())

    def setChargeOnGrid(self, chargeOnGrid):
        self.chargeOnGrid = D.to_device(chargeOnGrid, torch.float64)

    def _field_table(self, gridObj, field, ncomp):
        f = D.to_device(field, torch.float64).reshape(-1)
        G = gridObj.getNpExt()
        if f.shape[0] < ncomp * G:
            raise ValueError(f"field must hold {ncomp}*npExt values")
        tab = D.empty(4 * ncomp * G, torch.float32)
        _lib.call("oec_field_prepare", gridObj.c_grid(), f.data_ptr(), ncomp, tab.data_ptr(), D.stream())
        return tab

    def eFieldToParticles(self, gridObj, eAtGridPoints):
        """particles.pyx:58-62: bilinear gather of [Ex | Ey] node fields."""
        self._bind(gridObj)
        self._etab = self._field_table(gridObj, eAtGridPoints, 2)
        self.eAtParticles = D.empty((max(self._cap, 1), 2), torch.float64)
        _lib.call("oec_gather", gridObj.c_grid(), self.c_particles(), self._etab.data_ptr(), 2,
                  self.eAtParticles.data_ptr(), D.stream())

    def bFieldToParticles(self, gridObj, bAtGridPoints):
        """particles.pyx:64-68: bilinear gather of [Bx | By | Bz] node fields."""
        self._bind(gridObj)
        self._btab = self._field_table(gridObj, bAtGridPoints, 3)
        self.bAtParticles = D.empty((max(self._cap, 1), 3), torch.float64)
        _lib.call("oec_gather", gridObj.c_grid(), self.c_particles(), self._btab.data_ptr(), 3,
                  self.bAtParticles.data_ptr(), D.stream())

    def getEAtParticles(self):
        n = self.getMacroParticleCount()
        return D.to_numpy(self.eAtParticles[:n])

    def getBAtParticles(self):
        n = self.getMacroParticleCount()
        return D.to_numpy(self.bAtParticles[:n])

    def borisPush(self, dt, typeBField=2):
        """particles.pyx:79-92: typeBField 0 (no B), 1 (constant B), 2 (gathered B)."""
        if self.eAtParticles is None:
            raise RuntimeError("eFieldToParticles must be called before borisPush")
        self.dt = float(dt)
        typeBField = int(typeBField)
        b_at = None
        if typeBField == 2:
            if self.bAtParticles is None:
                raise RuntimeError("bFieldToParticles must be called before borisPush(typeBField=2)")
            b_at = self.bAtParticles.data_ptr()
        _lib.call("oec_boris_push", self._grid.c_grid(), self.c_particles(), self.eAtParticles.data_ptr(), b_at,
                  _lib.d3(self.bConst), self.dt, self.particleCharge / self.particleMass, typeBField, D.stream())

    def _hole_buffers(self):
        if getattr(self, "_holes", None) is None or self._holes.shape[0] < self._cap:
            self._holes = D.empty(max(self._cap, 1), torch.int32)
            self._n_holes = D.zeros(1, torch.int32)
            self._scan_scratch = D.zeros(1024, torch.int32)
            self._n_add = D.zeros(1, torch.int32)

    def addAndRemoveParticles(self, addParticleData, keepParticles=None, deposit=False):
        """particles.pyx:94-121: drop the particles with keepParticles == 0 and
        insert the rows of addParticleData (device tensor or numpy (n, 6)).

        keepParticles: u16 per particle (1 = keep), or None to use the
        absorbed bits of the last inside test already on the device.  Every
        particle lands in the slot the reference gives it (oec_add_remove
        follows the reference's three placement rules, with the row count of
        its array tracked on the device)."""
        n_old = self.getMacroParticleCount()
        if keepParticles is not None:
            keep = D.to_device(np.asarray(keepParticles, dtype=np.uint16).astype(np.int16), torch.int16)
            if keep.shape[0] < n_old:
                raise ValueError("keepParticles must have one entry per particle")
            _lib.call("oec_mask_from_keep", keep.data_ptr(), n_old, self._mask.data_ptr(), self._mask.shape[0],
                      D.stream())
        add = addParticleData
        if not isinstance(add, torch.Tensor):
            add = np.ascontiguousarray(add, dtype=np.float64).reshape(-1, 6)
        n_add = int(add.shape[0])
        self._hole_buffers()
        p, s = self.c_particles(), D.stream()
        _lib.call("oec_absorbed_index", p, self._mask.data_ptr(), self._holes.data_ptr(), self._holes.shape[0],
                  self._n_holes.data_ptr(), self._scan_scratch.data_ptr(), None, s)
        n_holes = int(self._n_holes.item())
        n_new = n_old - n_holes + n_add
        if n_new > self._cap:
            self.ensure_capacity(int(n_new * 1.1) + 1)
            self._hole_buffers()
            p = self.c_particles()
            _lib.call("oec_absorbed_index", p, self._mask.data_ptr(), self._holes.data_ptr(), self._holes.shape[0],
                      self._n_holes.data_ptr(), self._scan_scratch.data_ptr(), None, s)
        add_dev = D.to_device(add, torch.float64).reshape(-1, 6) if n_add else D.zeros((1, 6), torch.float64)
        self._n_add.fill_(n_add)
        rho = wsc = None
        if deposit:
            self._deposit_buffers(self._grid)
            rho, wsc = self._rho_fix.data_ptr(), self._wscale.data_ptr()
        _lib.call("oec_add_remove", self._grid.c_grid(), p, self.c_scratch(), self._mask.data_ptr(),
                  self._holes.data_ptr(), self._n_holes.data_ptr(), self._holes.shape[0], add_dev.data_ptr(),
                  self._n_add.data_ptr(), max(n_add, 0), self._array_len.data_ptr(), rho, wsc,
                  self._status.data_ptr(), s)
        self.eAtParticles = None
        self.bAtParticles = None

    # ------------------------------------------------------- fused hot path
    def pushGatherDeposit(self, gridObj, eCellTable, dt, typeBField, boundary, deposit=True, bCellTable=None,
                          refreshScale=True):
        """One fused pass: gather E (and B), Boris push, move, inside test of
        `boundary`, absorbed bits, and (deposit=True) the int64 fixed-point
        deposit of the surviving particles for the next step's solve.

        eCellTable: device float32 cell-centric E table (``fieldTable``).
        refreshScale=False keeps the fixed-point scale of the previous call
        (valid while no weight has grown)."""
        self._bind(gridObj)
        self.dt = float(dt)
        g, p, s = gridObj.c_grid(), self.c_particles(), D.stream()
        rho = None
        if deposit:
            self._deposit_buffers(gridObj)
            if refreshScale:
                _lib.call("oec_deposit_scale", p, self._wscale.data_ptr(), s)
            rho = self._rho_fix.data_ptr()
        _lib.call("oec_push_gather", g, p, eCellTable.data_ptr(),
                  bCellTable.data_ptr() if bCellTable is not None else None, _lib.d3(self.bConst), self.dt,
                  self.particleCharge / self.particleMass, int(typeBField), boundary.c_boundary(),
                  self._mask.data_ptr(), rho, self._wscale.data_ptr(), self._status.data_ptr(), s)

    def fieldTable(self, gridObj, nodeField, ncomp=2):
        """Cell-centric float32 table of a node field for the fused kernel."""
        self._bind(gridObj)
        return self._field_table(gridObj, nodeField, ncomp)

    # ------------------------------------------------------------ inside
    def absorbedMask(self):
        return self._mask

    def getFullIsInside(self):
        return self.getIsInside()

    def getIsInside(self):
        """u16 per particle, 1 = inside (from the device absorbed bits)."""
        n = self.getMacroParticleCount()
        words = D.to_numpy(self._mask).view(np.uint32)
        bits = np.unpackbits(words.view(np.uint8), bitorder="little")[:n]
        return (1 - bits).astype(np.uint16)

    def status(self):
        st = D.to_numpy(self._status)
        return {k: int(st[i]) for i, k in enumerate(_lib.STATUS_FIELDS)}

    def clearStatus(self):
        self._status.zero_()
