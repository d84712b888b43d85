"""Device-resident integral data of one molecule and the calls on it.

An :class:`IntegralEngine` owns, on one CUDA device:

* the shell arrays (centres, momenta, primitive exponents and
  coefficient x normalisation products),
* every shell pair (i >= j, the reference's ``pair_list``, shelled.py:962-964)
  in canonical orientation l_a >= l_b, split into the pair classes ss/ps/pp and
  sorted by descending Schwarz factor, with SoA primitive-pair records and
  packed core records,
* the candidate-quartet queue: per quartet class, bra row r pairs with the
  ket prefix whose Schwarz product clears ``tau_schwarz``,
* with d shells: the pairs holding a d shell and every s/p pair again in the
  generic record layout, and the two candidate spaces (d pair | s/p pair),
  (d pair | d pair) that dftk_jk_hl adds to the s/p build,
* the J/K workspace.

Generally contracted shells enter the kernels as one shell per contraction
row (basis.segments); matrices keep the reference's AO order.

PyTorch only provides the device buffers and the stream; all arithmetic is in
``libdftk.so``.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib, basis as _basis

# quartet class of (bra pair class, ket pair class), bra class >= ket class
QCLASS_OF = {(0, 0): 0, (1, 0): 1, (1, 1): 2, (2, 0): 3, (2, 1): 4, (2, 2): 5}
QCLASS_PAIRS = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
QCLASS_NAMES = ["(ss|ss)", "(ps|ss)", "(ps|ps)", "(pp|ss)", "(pp|ps)", "(pp|pp)"]
PAIR_FIELDS = {0: 6, 1: 10, 2: 13}  # stored record fields per pair class (ERI fields + alpha)
GENERIC_FIELDS = 13  # the d-shell path's pair sets: every ERI field + alpha
# Fixed flop accounting per evaluated primitive quartet, by class (ss|ss)..(pp|pp):
# 2 x (R-recursion FMAs + ket Hermite contraction + bra contraction) + 40 + 3L.
FLOPS_PER_PRIM_QUARTET = [44, 66, 145, 147, 410, 1402]


def candidate_offsets(q_bra: np.ndarray, q_ket: np.ndarray, same_class: bool, tau: float) -> np.ndarray:
    """Row offsets of the candidate-quartet space of one quartet class.

    Both Schwarz-factor arrays are sorted in descending order, so bra row r
    keeps the ket prefix k < count_r with q_ket[k] >= tau / q_bra[r]; for
    bra class == ket class the prefix also stops at k <= r so each unique
    quartet appears once.  Returns int64 offsets of length n_rows + 1."""
    nrows = q_bra.size
    if nrows == 0 or q_ket.size == 0:
        return np.zeros(nrows + 1, dtype=np.int64)
    with np.errstate(divide="ignore"):
        thr = np.where(q_bra > 0, tau / np.where(q_bra > 0, q_bra, 1.0), np.inf)
    cnt = np.searchsorted(-q_ket, -thr, side="right").astype(np.int64)
    if same_class:
        cnt = np.minimum(cnt, np.arange(1, nrows + 1))
    return np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)


def hlc_bucket(nprim: np.ndarray) -> np.ndarray:
    """Primitive-pair-count bucket of each pair (DFTK_HLC_BUCKET_BOUNDS)."""
    return np.searchsorted(np.asarray(_lib.HLC_BUCKET_BOUNDS), nprim, side="left").clip(0, _lib.HLC_NB - 1)


def hlc_spaces(l, nprim, hi_ab, lo_ab, q_hi, q_lo, tau):
    """Candidate spaces of the thread-per-quartet d classes (the layout
    dftk_hl_t documents): bra lists per hi kind (Schwarz order), ket lists
    per pair kind grouped by primitive-count bucket with their segment
    starts, and per class the offsets over (bra position, bucket): each
    segment's Schwarz prefix, cut at kets whose hi row is <= the bra's for a
    class whose two kinds are equal."""
    nb = _lib.HLC_NB
    sets = []
    for (a, b), q in ((lo_ab, q_lo), (hi_ab, q_hi)):
        la, lb = l[a], l[b]
        kind = np.where(la > 2, -1, np.where(la == 0, 0, np.where(la == 1, 1 + lb, 3 + lb)))
        sets.append((kind, hlc_bucket(nprim[a].astype(np.int64) * nprim[b]), q))
    rows = [np.nonzero(sets[1][0] == 3 + x)[0].astype(np.int32) for x in range(3)]
    kets, seg = [], []
    for y in range(6):
        kind, bucket, _ = sets[0 if y < 3 else 1]
        idx = np.nonzero(kind == y)[0]
        order = np.argsort(bucket[idx], kind="stable")
        kets.append(idx[order].astype(np.int32))
        seg.append(np.searchsorted(bucket[idx][order], np.arange(nb + 1), side="left").astype(np.int64))
    offs = []
    for bk, kk in _lib.HLC_CLASS_KINDS:
        bra = rows[bk - 3]
        qk = sets[0 if kk < 3 else 1][2]
        with np.errstate(divide="ignore"):
            qb = q_hi[bra]
            thr = np.where(qb > 0, tau / np.where(qb > 0, qb, 1.0), np.inf)
        cnt = np.zeros((bra.size, nb), dtype=np.int64)
        for b in range(nb):
            segk = kets[kk][seg[kk][b]:seg[kk][b + 1]]
            c = np.searchsorted(-qk[segk], -thr, side="right")
            if bk == kk:
                c = np.minimum(c, np.searchsorted(segk, bra, side="right"))
            cnt[:, b] = np.where(qb > 0, c, 0)
        offs.append(np.concatenate([[0], np.cumsum(cnt.reshape(-1))]).astype(np.int64))
    return rows, kets, seg, offs


def shard_row_offsets(row_off: np.ndarray, rank: int, world: int) -> np.ndarray:
    """Row offsets of one rank's share of a class's candidate space.

    Rows are split into `world` contiguous ranges holding equal numbers of
    candidates (the range of rank r starts at the first row whose offset
    reaches r/world of the total); rows outside the rank's range keep zero
    candidates, so the kernels take the shard unchanged and every candidate
    belongs to exactly one rank."""
    off = np.asarray(row_off, dtype=np.int64)
    total = int(off[-1])
    n_rows = off.size - 1
    bounds = [int(np.searchsorted(off[:-1], total * r // world, side="left")) if r < world else n_rows
              for r in range(world + 1)]
    bounds[0] = 0
    lo, hi = bounds[rank], bounds[rank + 1]
    cnt = np.diff(off)
    mine = np.zeros_like(cnt)
    mine[lo:hi] = cnt[lo:hi]
    return np.concatenate([[0], np.cumsum(mine)]).astype(np.int64)


def _dev(device) -> torch.device:
    if device is None:
        if not torch.cuda.is_available():
            raise _lib.DftkError("engine", _lib.ERR_CUDA, "no CUDA device: the integral engine has no CPU path")
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device(device)


class IntegralEngine:
    def __init__(self, shells: List[Dict], tau_schwarz: float = 1e-12, tau_prim: float = 1e-15, device=None,
                 hl_classes: bool = True):
        _basis.check_supported(shells)
        # (ds|..) and (dp|..) quartets with s/p kets through the generated
        # thread-per-quartet kernels (False: every d quartet through the
        # warp-per-quartet kernel)
        self.hl_classes = bool(hl_classes)
        _lib.load()
        self.device = _dev(device)
        self.shells = shells
        # integral shells: one per contraction row (basis.segments); equal to
        # the shells unless a shell is generally contracted
        self.segs = _basis.segments(shells)
        self.general = len(self.segs) != len(shells)
        self.ns = len(self.segs)
        self.n_ao = int(shells[-1]["ao_stop"]) if shells else 0
        self.tau_schwarz = float(tau_schwarz)
        self.tau_prim = float(tau_prim)
        self.l = np.array([s["l"] for s in self.segs], dtype=np.int32)
        self.nao_sh = np.array([s["n_ao"] for s in shells], dtype=np.int64)  # per reference shell
        self.has_hl = bool((self.l >= 2).any())
        with torch.cuda.device(self.device):
            _lib.call("dftk_init")
            self._upload_shells()
            self._build_pairs()
            self._build_queue()
            if self.has_hl:
                self._build_hl()
            nbytes = _lib.load().dftk_jk_workspace_bytes_queue(self.ns, self.n_ao, ctypes.byref(self.c_queue))
            self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
            self.workspace_bytes = int(nbytes)
            self.base_workspace_bytes = int(_lib.load().dftk_jk_workspace_bytes(self.ns, self.n_ao))

    # ------------------------------------------------------------------ setup
    def _t(self, arr, dtype):
        return torch.as_tensor(np.ascontiguousarray(arr), dtype=dtype).to(self.device)

    def _upload_shells(self):
        sh = self.segs
        nprim = np.array([s["exponents"].size for s in sh], dtype=np.int32)
        self._seg_nprim = nprim
        prim_off = np.concatenate([[0], np.cumsum(nprim)[:-1]]).astype(np.int32)
        exps = np.concatenate([s["exponents"] for s in sh]) if sh else np.zeros(0)
        # coefficient x radial norm per primitive (for s and p shells this is
        # normal() itself; d components get their remaining factor in-kernel)
        cn = np.concatenate([s["cn"] for s in sh]) if sh else np.zeros(0)
        self.kmax = int(max(1, (nprim.max() if sh else 1) ** 2))
        self.d_xyz = self._t(np.array([s["atom_pos"] for s in sh], dtype=np.float64).reshape(-1), torch.float64)
        self.d_l = self._t(self.l, torch.int32)
        self.d_nprim = self._t(nprim, torch.int32)
        self.d_prim_off = self._t(prim_off, torch.int32)
        self.d_ao = self._t(np.array([s["ao_start"] for s in sh], dtype=np.int32), torch.int32)
        if self.kmax > 128:
            raise _basis.UnsupportedBasis(f"{int(nprim.max())} primitives in one contraction (at most 11)")
        self.d_exp = self._t(exps.astype(np.float64), torch.float64)
        self.d_cn = self._t(cn.astype(np.float64), torch.float64)
        self.c_shells = _lib.Shells(
            self.ns, self.n_ao, _lib.ptr(self.d_xyz).value, _lib.ptr(self.d_l).value, _lib.ptr(self.d_nprim).value,
            _lib.ptr(self.d_prim_off).value, _lib.ptr(self.d_ao).value, _lib.ptr(self.d_exp).value,
            _lib.ptr(self.d_cn).value)

    def _alloc_class(self, pc: int, ab: np.ndarray):
        n = ab.shape[0]
        nf = PAIR_FIELDS.get(pc, GENERIC_FIELDS)
        bufs = {
            "ab": self._t(ab.reshape(-1).astype(np.int32), torch.int32) if n else torch.zeros(2, dtype=torch.int32, device=self.device),
            "nprim": torch.zeros(max(n, 1), dtype=torch.int32, device=self.device),
            "rec64": torch.zeros(max(nf * self.kmax * n, 1), dtype=torch.float64, device=self.device),
            "rec32": torch.zeros(max(nf * self.kmax * n, 1), dtype=torch.float32, device=self.device),
            "q": torch.zeros(max(n, 1), dtype=torch.float64, device=self.device),
            "qp": torch.zeros(max(self.kmax * n, 1), dtype=torch.float32, device=self.device),
        }
        core = pc in PAIR_FIELDS  # packed core records: the s/p class kernels' inner loops read them
        if core:
            bufs["core64"] = torch.zeros(max(8 * self.kmax * n, 8), dtype=torch.float64, device=self.device)
            bufs["core32"] = torch.zeros(max(8 * self.kmax * n, 8), dtype=torch.float32, device=self.device)
        st = _lib.Pairs(n, self.kmax, _lib.ptr(bufs["ab"]).value, _lib.ptr(bufs["nprim"]).value,
                        _lib.ptr(bufs["rec64"]).value, _lib.ptr(bufs["rec32"]).value, _lib.ptr(bufs["q"]).value,
                        _lib.ptr(bufs["qp"]).value, _lib.ptr(bufs["core64"]).value if core else None,
                        _lib.ptr(bufs["core32"]).value if core else None)
        return bufs, st

    def _build_pairs(self):
        ns = self.ns
        ii, jj = np.tril_indices(ns)  # reference pair_list order: (i, j), j <= i
        ii = ii.astype(np.int64)
        jj = jj.astype(np.int64)
        swap = self.l[ii] < self.l[jj]
        a = np.where(swap, jj, ii)
        b = np.where(swap, ii, jj)
        # s/p pairs by l_a + l_b; pairs with a d shell (class 3) go to _build_hl
        pclass = np.where(self.l[a] >= 2, 3, self.l[a] + self.l[b])
        self._pair_a, self._pair_b, self._pair_class = a, b, pclass
        stream = _lib.stream_handle()
        self.pair_bufs, self.c_pairs_list = [], []
        ref_class = np.zeros(ii.size, dtype=np.int32)
        ref_row = np.zeros(ii.size, dtype=np.int64)
        self.q_sorted = []
        for pc in range(3):
            sel = np.nonzero(pclass == pc)[0]
            ab = np.stack([a[sel], b[sel]], axis=1)
            bufs, st = self._alloc_class(pc, ab)
            if ab.shape[0]:
                _lib.call("dftk_pair_data", ctypes.byref(self.c_shells), pc, ctypes.byref(st), stream)
                _lib.call("dftk_schwarz", ctypes.byref(self.c_shells), pc, ctypes.byref(st), stream)
                q = bufs["q"][: ab.shape[0]].cpu().numpy()
                order = np.argsort(-q, kind="stable")
                ab = ab[order]
                sel = sel[order]
                bufs, st = self._alloc_class(pc, ab)
                _lib.call("dftk_pair_data", ctypes.byref(self.c_shells), pc, ctypes.byref(st), stream)
                _lib.call("dftk_schwarz", ctypes.byref(self.c_shells), pc, ctypes.byref(st), stream)
                self.q_sorted.append(bufs["q"][: ab.shape[0]].cpu().numpy())
            else:
                self.q_sorted.append(np.zeros(0))
            ref_class[sel] = pc
            ref_row[sel] = np.arange(sel.size)
            self.pair_bufs.append(bufs)
            self.c_pairs_list.append(st)
        self.c_pairs = _lib.PairsArray(*self.c_pairs_list)
        ref_class[pclass == 3] = 3  # rows of these pairs are set by _build_hl
        # reference pair index i(i+1)/2 + j -> (class, sorted row, stored as (j, i))
        self.ref_pair_class = ref_class
        self.ref_pair_row = ref_row
        self.ref_pair_swap = swap
        self.n_pairs = [int(x.shape[0]) for x in self.q_sorted]

    def _build_queue(self):
        self.row_off = []
        self.totals = []
        q = _lib.Queue()
        for c, (X, Y) in enumerate(QCLASS_PAIRS):
            qx, qy = self.q_sorted[X], self.q_sorted[Y]
            nrows = qx.size
            off = candidate_offsets(qx, qy, X == Y, self.tau_schwarz)
            d_off = self._t(off, torch.int64)
            self.row_off.append(d_off)
            self.totals.append(int(off[-1]))
            q.n_rows[c] = nrows if off[-1] > 0 else 0
            q.total[c] = int(off[-1])
            q.row_off[c] = _lib.ptr(d_off).value
        q.tau_prim = self.tau_prim
        # group selected quartets by the ket's primitive-count bucket when the
        # s/p pairs differ in primitive count (general contractions)
        sp = self._pair_class < 3
        pb = hlc_bucket(self._seg_nprim[self._pair_a[sp]].astype(np.int64) * self._seg_nprim[self._pair_b[sp]])
        q.bucket_kets = int(np.unique(pb).size > 1)
        self.c_queue = q

    def _generic_set(self, sel: np.ndarray):
        """Pairs `sel` (indices into the pair list) in the generic 13-field
        layout, sorted by descending Schwarz factor: (buffers, struct, q, sel)."""
        a, b = self._pair_a, self._pair_b
        stream = _lib.stream_handle()
        ab = np.stack([a[sel], b[sel]], axis=1)
        bufs, st = self._alloc_class(_lib.PCLASS_GENERIC, ab)
        if ab.shape[0] == 0:
            return bufs, st, np.zeros(0), sel
        for _ in range(2):  # measure, sort, then build the sorted set
            _lib.call("dftk_pair_data", ctypes.byref(self.c_shells), _lib.PCLASS_GENERIC, ctypes.byref(st), stream)
            _lib.call("dftk_hl_schwarz", ctypes.byref(self.c_shells), ctypes.byref(st), self.hl_lmax, stream)
            q = bufs["q"][: ab.shape[0]].cpu().numpy()
            if _ == 1:
                break
            order = np.argsort(-q, kind="stable")
            ab, sel = ab[order], sel[order]
            bufs, st = self._alloc_class(_lib.PCLASS_GENERIC, ab)
        return bufs, st, q, sel

    def _build_hl(self):
        """Pair sets and candidate spaces of the quartets with a d shell:
        rows are the d pairs; kets the s/p pairs ((hi|lo)) or the d pairs up
        to the row ((hi|hi)), each a Schwarz prefix as in the s/p queue."""
        pclass = self._pair_class
        self.hl_lmax = int(self.l.max())
        hi_bufs, hi_st, q_hi, sel_hi = self._generic_set(np.nonzero(pclass == 3)[0])
        lo_bufs, lo_st, q_lo, sel_lo = self._generic_set(np.nonzero(pclass < 3)[0])
        self.ref_pair_row[sel_hi] = np.arange(sel_hi.size)
        self.ref_pair_lo_row = np.full(pclass.size, -1, dtype=np.int64)
        self.ref_pair_lo_row[sel_lo] = np.arange(sel_lo.size)
        off_lo = candidate_offsets(q_hi, q_lo, False, self.tau_schwarz)
        off_hi = candidate_offsets(q_hi, q_hi, True, self.tau_schwarz)
        spaces = hlc_spaces(self.l, self._seg_nprim, (self._pair_a[sel_hi], self._pair_b[sel_hi]),
                            (self._pair_a[sel_lo], self._pair_b[sel_lo]), q_hi, q_lo, self.tau_schwarz)
        self.hlc_rows, self.hlc_kets, self.hlc_seg, hlc_off = spaces
        if self.hl_classes:
            # rows whose every (hi|lo) quartet belongs to a class leave the
            # warp kernel's (hi|lo) space
            cnt = np.diff(off_lo)
            for x in range(3):
                if sum(1 for bk, kk in _lib.HLC_CLASS_KINDS if bk == x + 3 and kk < 3) == 3:
                    cnt[self.hlc_rows[x]] = 0
            off_lo = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
            # (hi|hi) likewise, for rows of a kind that has a class with every
            # hi kind, when no hi pair has an f shell
            if self.hl_lmax <= 2:
                cnt = np.diff(off_hi)
                for x in range(3):
                    n = sum(1 for bk, kk in _lib.HLC_CLASS_KINDS
                            if (bk == x + 3 and kk >= 3) or (kk == x + 3 and bk >= 3 and bk != kk))
                    if n == 3:
                        cnt[self.hlc_rows[x]] = 0
                off_hi = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
        else:
            hlc_off = [np.zeros(1, dtype=np.int64) for _ in hlc_off]
        self.hlc_totals = [int(o[-1]) for o in hlc_off]
        self.hl_bufs = (hi_bufs, lo_bufs)
        self.hl_row_off = (self._t(off_lo, torch.int64), self._t(off_hi, torch.int64))
        self.hl_q = (q_hi, q_lo)
        self.hl_totals = [int(off_lo[-1]), int(off_hi[-1])]
        hl = _lib.HlSet()
        hl.hi = hi_st
        hl.lo = lo_st
        hl.n_rows = int(q_hi.size)
        for k in range(2):
            hl.total[k] = self.hl_totals[k]
            hl.row_off[k] = _lib.ptr(self.hl_row_off[k]).value
        hl.tau_prim = self.tau_prim
        hl.lmax = self.hl_lmax
        if self.hl_classes:
            self.hlc_dev = ([self._t(r, torch.int32) if r.size else None for r in self.hlc_rows],
                            [self._t(k, torch.int32) if k.size else None for k in self.hlc_kets],
                            [self._t(o, torch.int64) for o in hlc_off])
            for x in range(3):
                if self.hlc_rows[x].size:
                    hl.cls_rows[x] = _lib.ptr(self.hlc_dev[0][x]).value
                    hl.n_cls_rows[x] = int(self.hlc_rows[x].size)
            for y in range(6):
                if self.hlc_kets[y].size:
                    hl.cls_kets[y] = _lib.ptr(self.hlc_dev[1][y]).value
                for b in range(_lib.HLC_NB + 1):
                    hl.cls_ket_seg[y][b] = int(self.hlc_seg[y][b])
            for c in range(_lib.HLC_N_CLASSES):
                hl.cls_off[c] = _lib.ptr(self.hlc_dev[2][c]).value
                hl.cls_total[c] = self.hlc_totals[c]
        self.c_hl = hl

    # ---------------------------------------------------------------- queries
    def quartet_totals(self) -> List[int]:
        """Schwarz-surviving unique quartets per class (ss|ss)..(pp|pp)."""
        return list(self.totals)

    @staticmethod
    def fixed_flops(prim_counts: Sequence[int]) -> float:
        """Fixed-accounting flops of `prim_counts` evaluated primitive quartets per class."""
        return float(sum(FLOPS_PER_PRIM_QUARTET[c] * prim_counts[c] for c in range(6)))

    # ---------------------------------------------------------------- compute
    def one_electron(self, atoms: Sequence[str], centers) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """S, T, V as N x N float64 CUDA tensors."""
        N = self.n_ao
        xyz = torch.as_tensor(np.asarray(centers, dtype=np.float64).reshape(-1), device=self.device)
        z = torch.as_tensor(np.array([float(int(a)) for a in atoms]), dtype=torch.float64, device=self.device)
        S, T, V = (torch.empty((N, N), dtype=torch.float64, device=self.device) for _ in range(3))
        _lib.call("dftk_one_electron", ctypes.byref(self.c_shells), len(atoms), _lib.ptr(xyz), _lib.ptr(z),
                  _lib.ptr(S), _lib.ptr(T), _lib.ptr(V), _lib.stream_handle())
        return S, T, V

    def shard_queue(self, rank: int, world: int):
        """A queue holding this rank's share of every class's candidates
        (shard_row_offsets); pass it to jk(queue=...) and sum the partial J/K
        over the ranks."""
        q = _lib.Queue()
        keep = []
        for c in range(len(QCLASS_PAIRS)):
            off = shard_row_offsets(self.row_off[c].cpu().numpy(), rank, world)
            d_off = self._t(off, torch.int64)
            keep.append(d_off)
            q.n_rows[c] = self.c_queue.n_rows[c] if off[-1] > 0 else 0
            q.total[c] = int(off[-1])
            q.row_off[c] = _lib.ptr(d_off).value
            q.ket_base[c] = self.c_queue.ket_base[c]
        q.tau_prim = self.c_queue.tau_prim
        q.mol_active = self.c_queue.mol_active
        q.bucket_kets = self.c_queue.bucket_kets
        q._keep = keep  # device arrays live as long as the queue
        return q

    def jk(self, D: torch.Tensor, D_a: Optional[torch.Tensor] = None, D_b: Optional[torch.Tensor] = None,
           uhf: bool = False, mixed: bool = False, tau: float = 1e-14, tau_fp32: float = 1e-6,
           out=None, counts: Optional[torch.Tensor] = None, scan: bool = False, queue=None,
           persist: bool = False):
        """Direct J, K_a (, K_b) for densities on the device.

        D is the density J is built from (the reference's P = P_a + P_b);
        K_a uses D_a (defaults to D / 2, the RHF alpha density) and, with
        ``uhf``, K_b uses D_b.  Returns (J, K_a, K_b) with K_b = K_a unless uhf.
        ``scan`` hands dftk_jk only the base workspace, which selects its
        direct path (class kernels scan the candidates themselves) instead of
        the selection pass + quartet lists; ``persist`` runs the list path as
        one selection launch and one persistent launch per precision
        (DFTK_JK_PERSIST).
        """
        N = self.n_ao
        dev = self.device
        D = self._square(D)
        D_a = self._square(D_a) if D_a is not None else (0.5 * D).contiguous()
        if uhf:
            if D_b is None:
                raise _lib.DftkError("jk", _lib.ERR_ARG, "uhf needs D_b")
            D_b = self._square(D_b)
        if out is None:
            J = torch.empty((N, N), dtype=torch.float64, device=dev)
            Ka = torch.empty((N, N), dtype=torch.float64, device=dev)
            Kb = torch.empty((N, N), dtype=torch.float64, device=dev) if uhf else None
        else:
            J, Ka, Kb = out
        flags = (_lib.JK_UHF if uhf else 0) | (_lib.JK_MIXED if mixed else 0) | (_lib.JK_PERSIST if persist else 0)
        if self.has_hl and queue is not None:
            raise _basis.UnsupportedBasis("jk(queue=...): sharded builds cover s/p bases")
        _lib.call("dftk_jk", ctypes.byref(self.c_shells), self.c_pairs,
                  ctypes.byref(queue if queue is not None else self.c_queue),
                  _lib.ptr(D), _lib.ptr(D_a), _lib.ptr(D_b if uhf else None), _lib.ptr(J), _lib.ptr(Ka),
                  _lib.ptr(Kb if uhf else None), flags, float(tau), float(tau_fp32 if mixed else tau),
                  _lib.ptr(self.workspace), self.base_workspace_bytes if scan else self.workspace_bytes,
                  _lib.ptr(counts), _lib.stream_handle())
        if self.has_hl:
            # quartets with a d shell (FP64), added to the s/p part
            _lib.call("dftk_jk_hl", ctypes.byref(self.c_shells), ctypes.byref(self.c_hl), _lib.ptr(D), _lib.ptr(D_a),
                      _lib.ptr(D_b if uhf else None), _lib.ptr(J), _lib.ptr(Ka), _lib.ptr(Kb if uhf else None),
                      _lib.JK_UHF if uhf else 0, float(tau), _lib.ptr(self.workspace), self.workspace_bytes, None,
                      _lib.stream_handle())
        return J, Ka, (Kb if uhf else Ka)

    def _square(self, M) -> torch.Tensor:
        if not isinstance(M, torch.Tensor):
            M = torch.as_tensor(np.asarray(M, dtype=np.float64))
        M = M.to(device=self.device, dtype=torch.float64).contiguous()
        if M.shape != (self.n_ao, self.n_ao):
            raise _lib.DftkError("jk", _lib.ERR_ARG, f"density shape {tuple(M.shape)} != ({self.n_ao}, {self.n_ao})")
        return M

    def gradient(self, atoms: Sequence[str], centers, D: torch.Tensor, D_a: torch.Tensor, D_b: torch.Tensor,
                 W: torch.Tensor, tau: float = 1e-14, tau_fp32: float = 0.0, scan: bool = False) -> np.ndarray:
        """Electronic nuclear gradient (n_atoms, 3): sum D dH - sum W dS + sum Gamma d(ERI),
        from the total density D, spin densities D_a/D_b and energy-weighted density W.
        tau_fp32 > tau selects the mixed form; ``scan`` hands dftk_grad only the
        base workspace (class kernels scan the candidates, FP64 only)."""
        if self.has_hl:
            raise _basis.UnsupportedBasis("gradient: the derivative kernels cover s and p shells")
        n_atoms = len(atoms)
        if not hasattr(self, "d_shell_atom"):
            self.d_shell_atom = self._t(np.array([s["atom_idx"] for s in self.segs], dtype=np.int32), torch.int32)
        xyz = torch.as_tensor(np.asarray(centers, dtype=np.float64).reshape(-1), device=self.device)
        z = torch.as_tensor(np.array([float(int(a)) for a in atoms]), dtype=torch.float64, device=self.device)
        g = torch.zeros(3 * n_atoms, dtype=torch.float64, device=self.device)
        _lib.call("dftk_grad", ctypes.byref(self.c_shells), _lib.ptr(self.d_shell_atom), n_atoms, _lib.ptr(xyz),
                  _lib.ptr(z), self.c_pairs, ctypes.byref(self.c_queue), _lib.ptr(self._square(D)),
                  _lib.ptr(self._square(D_a)), _lib.ptr(self._square(D_b)), _lib.ptr(self._square(W)), float(tau),
                  float(tau_fp32), _lib.ptr(g), _lib.ptr(self.workspace),
                  self.base_workspace_bytes if scan else self.workspace_bytes, _lib.stream_handle())
        return g.reshape(n_atoms, 3).cpu().numpy()

    def quartet_descriptors(self, quads: np.ndarray):
        """Map reference quartets (a, b, c, d) to dftk_eri_blocks descriptors and offsets."""
        quads = np.asarray(quads, dtype=np.int64).reshape(-1, 4)
        a, b, c, d = quads.T

        def pair_info(x, y):
            i = np.maximum(x, y)
            j = np.minimum(x, y)
            idx = i * (i + 1) // 2 + j
            pc = self.ref_pair_class[idx]
            row = self.ref_pair_row[idx]
            # canonical first shell: i unless swapped to (j, i)
            first = np.where(self.ref_pair_swap[idx], j, i)
            flip = (first != x).astype(np.int32)
            return pc, row, flip

        pc1, r1, f1 = pair_info(a, b)
        pc2, r2, f2 = pair_info(c, d)
        exch = pc1 < pc2
        X = np.where(exch, pc2, pc1)
        Y = np.where(exch, pc1, pc2)
        rb = np.where(exch, r2, r1)
        rk = np.where(exch, r1, r2)
        fb = np.where(exch, f2, f1)
        fk = np.where(exch, f1, f2)
        qc = np.array([QCLASS_OF[(int(x), int(y))] for x, y in zip(X, Y)], dtype=np.int32) if quads.shape[0] else \
            np.zeros(0, dtype=np.int32)
        flags = fb | (fk << 1) | (exch.astype(np.int32) << 2)
        desc = np.stack([qc, rb.astype(np.int32), rk.astype(np.int32), flags.astype(np.int32)], axis=1)
        sizes = self.nao_sh[a] * self.nao_sh[b] * self.nao_sh[c] * self.nao_sh[d]
        off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        return desc.astype(np.int32), off

    def eri_blocks(self, quads: np.ndarray, fp32: bool = False) -> Tuple[torch.Tensor, np.ndarray]:
        """Contracted ERI blocks of reference quartets, flat in calc_eri layout
        (fp32=True evaluates the s/p quartets with the mixed path's FP32
        kernels; quartets with a d shell are always FP64)."""
        quads = np.asarray(quads, dtype=np.int64).reshape(-1, 4)
        if self.general:
            raise _basis.UnsupportedBasis("eri_blocks: generally contracted shells (use jk)")
        a, b, c, d = quads.T
        sizes = self.nao_sh[a] * self.nao_sh[b] * self.nao_sh[c] * self.nao_sh[d]
        off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        out = torch.zeros(int(off[-1]), dtype=torch.float64, device=self.device)
        hi = np.zeros(quads.shape[0], dtype=bool)
        if self.has_hl and quads.shape[0]:
            hi = (np.maximum(self.l[a], self.l[b]) >= 2) | (np.maximum(self.l[c], self.l[d]) >= 2)
        sp = np.nonzero(~hi)[0]
        if sp.size:
            desc, _ = self.quartet_descriptors(quads[sp])
            if fp32:
                desc[:, 3] |= 8
            d_desc = self._t(desc.reshape(-1), torch.int32)
            d_off = self._t(off[:-1][sp], torch.int64)
            _lib.call("dftk_eri_blocks", ctypes.byref(self.c_shells), self.c_pairs, desc.shape[0],
                      _lib.ptr(d_desc), _lib.ptr(d_off), _lib.ptr(out), _lib.stream_handle())
        hq = np.nonzero(hi)[0]
        if hq.size:
            desc = self._hl_descriptors(quads[hq])
            d_desc = self._t(desc.reshape(-1), torch.int32)
            d_off = self._t(off[:-1][hq], torch.int64)
            _lib.call("dftk_hl_eri_blocks", ctypes.byref(self.c_shells), ctypes.byref(self.c_hl), desc.shape[0],
                      _lib.ptr(d_desc), _lib.ptr(d_off), _lib.ptr(out), _lib.stream_handle())
        return out, off

    def _hl_descriptors(self, quads: np.ndarray) -> np.ndarray:
        """dftk_hl_eri_blocks descriptors of reference quartets with a d shell:
        the pair holding a d shell (the first one if both do) is the bra."""
        a, b, c, d = quads.T

        def pair_info(x, y):
            i = np.maximum(x, y)
            j = np.minimum(x, y)
            idx = i * (i + 1) // 2 + j
            is_hi = self.ref_pair_class[idx] == 3
            row = np.where(is_hi, self.ref_pair_row[idx], self.ref_pair_lo_row[idx])
            first = np.where(self.ref_pair_swap[idx], j, i)
            return is_hi, row, (first != x).astype(np.int32)

        h1, r1, f1 = pair_info(a, b)
        h2, r2, f2 = pair_info(c, d)
        exch = ~h1
        kind = (h1 & h2).astype(np.int32)
        rb = np.where(exch, r2, r1)
        rk = np.where(exch, r1, r2)
        fb = np.where(exch, f2, f1)
        fk = np.where(exch, f1, f2)
        flags = fb | (fk << 1) | (exch.astype(np.int32) << 2)
        n = self.nao_sh
        return np.stack([kind, rb, rk, flags, n[a], n[b], n[c], n[d]], axis=1).astype(np.int32)
