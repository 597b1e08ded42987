"""A CPU stand-in for one y-slab of the one-process-per-GPU protocol
(lagrangianrbnudging_b200.slabrank), for the gloo tests of the exchange.

Every rank steps the same whole domain with the oracle; its stand-in slab
holds the rows [j0, j0 + nyl) and the particles whose cell lies in them.  It
writes its messages in the library's byte layout (lbrb_slab_particle_format:
a 32-byte header, 80-byte hand-off records, moment planes from byte 256) and
checks every message it receives against the oracle's whole domain: the
ghost rows and moment rows must be its neighbours' rows of this step, and
after each receive its particles (those it kept and those handed to it, read
back from the received bytes) must equal the oracle's particles of the same
ids.  So a message sent to the wrong rank, into the wrong buffer, at the
wrong step or in the wrong layout fails the run."""
from __future__ import annotations

import numpy as np
import torch

from oracle.oracle import Oracle

HEADER = np.dtype([("count", "<i4"), ("step", "<i4"), ("j0", "<i4"), ("j1", "<i4"), ("kind", "<i4"),
                   ("pad", "<i4", (3,))])
RECORD = np.dtype([("P", "<f8", (9,)), ("id", "<i4"), ("type", "<i4")])
MOM_UP, MOM_DOWN, HAND_UP, HAND_DOWN = 1, 2, 3, 4
PLANES_OFF = 256
FIELDS = ["x", "y", "u", "v", "xo", "yo", "uo", "vo", "invtau"]


def cell_row(y: np.ndarray, ny: int) -> np.ndarray:
    """the cell row of positions (C truncation, periodic), as the kernels take it"""
    y = np.asarray(y, dtype=np.float64)
    ok = (y > -2.0) & (y < ny + 2.0)
    r = np.where(ok, np.trunc(np.where(ok, y, 0.0)).astype(np.int64) - 1, 0)
    return np.mod(r, ny)


class StandInSlab:
    def __init__(self, params: dict, j0: int, nyl: int, seed: int, particles: dict, xcap: int):
        self.nx, self.nyT = int(params["nx"]), int(params["ny"])
        self.j0, self.nyl, self.xcap = j0, nyl, xcap
        n = len(particles["id"])
        self.orc = Oracle(params, nprtcl=n)
        self.orc.init_conduction(seed, 2e-2)
        self.orc.set_particles(particles["id"], particles["x"], particles["y"], particles["u"], particles["v"],
                               particles["type"], particles["invtau"])
        self.istep = 0
        keep = self._mine(particles["y"])
        self.ids = np.asarray(particles["id"], np.int32)[keep]
        self.type = np.asarray(particles["type"], np.int32)[keep]
        self.P = np.stack([np.asarray(particles[k], np.float64)[keep]
                           for k in ("x", "y", "u", "v", "x", "y", "u", "v", "invtau")])
        self.handed = 0  # particles this slab handed to a neighbour
        nx = self.nx
        self.pstride = (nx * 8 + 255) // 256 * 256
        gb = 6 * nx * 8
        hb = HEADER.itemsize + xcap * RECORD.itemsize
        lo_wall, hi_wall = j0 == 0, j0 + nyl == self.nyT
        self.np_bufs = {
            "up": np.zeros(gb, np.uint8), "down": np.zeros(gb, np.uint8),
            "ghost_lo": None if lo_wall else np.zeros(gb, np.uint8),
            "ghost_hi": None if hi_wall else np.zeros(gb, np.uint8),
            "mom_up": np.zeros(PLANES_OFF + 3 * self.pstride, np.uint8),
            "mom_down": np.zeros(PLANES_OFF + 8 * self.pstride, np.uint8),
            "mom_lo": np.zeros(PLANES_OFF + 3 * self.pstride, np.uint8),
            "mom_hi": np.zeros(PLANES_OFF + 8 * self.pstride, np.uint8),
        }
        for k in ("hand_up", "hand_down", "hand_lo", "hand_hi"):
            self.np_bufs[k] = np.zeros(hb, np.uint8)
        self.bufs = {k: (None if a is None else torch.from_numpy(a)) for k, a in self.np_bufs.items()}

    # ---- helpers
    def _mine(self, y) -> np.ndarray:
        c = cell_row(y, self.nyT)
        return (c >= self.j0) & (c < self.j0 + self.nyl)

    def _row(self, j: int) -> int:
        return j % self.nyT

    def _ghost_up(self, j: int) -> np.ndarray:
        f, g = self.orc.f, self.orc.g
        return np.concatenate([f[2, j], f[5, j], f[6, j], g[2, j], g[5, j], g[6, j]]).view(np.uint8)

    def _ghost_down(self, j: int) -> np.ndarray:
        f, g = self.orc.f, self.orc.g
        return np.concatenate([f[4, j], f[7, j], f[8, j], g[4, j], g[7, j], g[8, j]]).view(np.uint8)

    def _write_mom(self, buf: np.ndarray, kind: int, planes) -> None:
        buf[:HEADER.itemsize] = np.array([(len(planes), self.istep, self.j0, self.j0 + self.nyl, kind,
                                           (0, 0, 0))], HEADER).view(np.uint8)
        for q, p in enumerate(planes):
            o = PLANES_OFF + q * self.pstride
            buf[o:o + self.nx * 8] = np.ascontiguousarray(p, np.float64).view(np.uint8)

    def _read_mom(self, buf: np.ndarray, nplanes: int):
        h = buf[:HEADER.itemsize].view(HEADER)[0]
        planes = [buf[PLANES_OFF + q * self.pstride:PLANES_OFF + q * self.pstride + self.nx * 8].view(np.float64)
                  for q in range(nplanes)]
        return h, planes

    def _rows_of(self, j: int, kinds):
        o = self.orc
        src = {"u": o.u, "v": o.v, "ub": o.ubef, "vb": o.vbef, "T": o.T}
        return [src[k][self._row(j)] for k in kinds]

    # ---- the slab interface SlabRank drives
    def slab_pack(self) -> None:
        top = self.j0 + self.nyl - 1
        self.np_bufs["up"][:] = self._ghost_up(top)
        self.np_bufs["down"][:] = self._ghost_down(self.j0)

    def step(self, n: int) -> None:
        assert n == 1
        # the ghost rows: the neighbours' boundary rows before this step
        if self.np_bufs["ghost_lo"] is not None:
            np.testing.assert_array_equal(self.np_bufs["ghost_lo"], self._ghost_up(self.j0 - 1))
        if self.np_bufs["ghost_hi"] is not None:
            np.testing.assert_array_equal(self.np_bufs["ghost_hi"], self._ghost_down(self.j0 + self.nyl))
        self.istep += 1
        self.orc.step(self.istep)

    def slab_moments_pack(self) -> None:
        top = self.j0 + self.nyl - 1
        self._write_mom(self.np_bufs["mom_up"], MOM_UP, self._rows_of(top, ("u", "v", "T")))
        self._write_mom(self.np_bufs["mom_down"], MOM_DOWN,
                        self._rows_of(self.j0, ("u", "v", "ub", "vb", "T"))
                        + self._rows_of(self.j0 + 1, ("u", "v", "T")))

    def slab_particles_step(self) -> None:
        nyT = self.nyT
        h, planes = self._read_mom(self.np_bufs["mom_lo"], 3)
        assert (h["kind"], h["step"], h["j1"] % nyT) == (MOM_UP, self.istep, self.j0), h
        for p, want in zip(planes, self._rows_of(self.j0 - 1, ("u", "v", "T"))):
            np.testing.assert_array_equal(p, want)
        h, planes = self._read_mom(self.np_bufs["mom_hi"], 8)
        assert (h["kind"], h["step"], h["j0"]) == (MOM_DOWN, self.istep, (self.j0 + self.nyl) % nyT), h
        want = (self._rows_of(self.j0 + self.nyl, ("u", "v", "ub", "vb", "T"))
                + self._rows_of(self.j0 + self.nyl + 1, ("u", "v", "T")))
        for p, w in zip(planes, want):
            np.testing.assert_array_equal(p, w)
        # advance: each own particle's state after this step is the oracle's
        idx = self._oracle_index(self.ids)
        self.P = np.stack([self.orc.pa[k][idx] for k in FIELDS])
        c = cell_row(self.P[1], nyT)
        up, down = c >= self.j0 + self.nyl, c < self.j0
        keep = ~(up | down)
        for name, sel, kind in (("hand_up", up, HAND_UP), ("hand_down", down, HAND_DOWN)):
            k = int(sel.sum())
            assert k <= self.xcap
            recs = np.zeros(k, RECORD)
            recs["P"] = self.P[:, sel].T
            recs["id"] = self.ids[sel]
            recs["type"] = self.type[sel]
            b = self.np_bufs[name]
            b[:HEADER.itemsize] = np.array([(k, self.istep, self.j0, self.j0 + self.nyl, kind, (0, 0, 0))],
                                           HEADER).view(np.uint8)
            b[HEADER.itemsize:HEADER.itemsize + k * RECORD.itemsize] = recs.view(np.uint8)
            self.handed += k
        self.P, self.ids, self.type = self.P[:, keep], self.ids[keep], self.type[keep]

    def slab_particles_recv(self) -> None:
        nyT = self.nyT
        got = []
        for name, kind, ok_rows in (("hand_lo", HAND_UP, lambda h: h["j1"] % nyT == self.j0),
                                    ("hand_hi", HAND_DOWN, lambda h: h["j0"] == (self.j0 + self.nyl) % nyT)):
            b = self.np_bufs[name]
            h = b[:HEADER.itemsize].view(HEADER)[0]
            assert h["kind"] == kind and h["step"] == self.istep and ok_rows(h), (name, h)
            k = int(h["count"])
            got.append(b[HEADER.itemsize:HEADER.itemsize + k * RECORD.itemsize].view(RECORD))
        for recs in got:
            self.P = np.concatenate([self.P, recs["P"].T], axis=1)
            self.ids = np.concatenate([self.ids, recs["id"]])
            self.type = np.concatenate([self.type, recs["type"]])
        # every particle now held, received bytes included, is the oracle's
        idx = self._oracle_index(self.ids)
        for q, k in enumerate(FIELDS):
            np.testing.assert_array_equal(self.P[q], self.orc.pa[k][idx])
        np.testing.assert_array_equal(self.type, self.orc.ptype[idx])
        assert np.all(self._mine(self.P[1]))

    def _oracle_index(self, ids) -> np.ndarray:
        oid = self.orc.pid[: self.orc.np]
        srt = np.argsort(oid)
        k = np.searchsorted(oid[srt], ids)
        assert np.all(oid[srt][k] == ids)
        return srt[k]
