"""Generate straight-line McMurchie-Davidson code for the s/p ERI classes.

Writes ``eri_classes.cuh`` next to this file.  Run it after changing the
class table; the generated header is committed so a build needs no Python.

For every angular class (La Lb | Lc Ld) with La >= Lb, Lc >= Ld and
La + Lb >= Lc + Ld (s = 0, p = 1) it emits one device function per
ket-component split.  The function evaluates the contracted Cartesian block
of one shell quartet from primitive-pair records:

    (ab|cd) = sum_{ij} sum_{tuv} E^{ab}_{tuv}(i) sum_{kl}
              sum_{tau nu phi} (-1)^{tau+nu+phi} E^{cd}_{tau nu phi}(kl) R_{t+tau,u+nu,v+phi}(i, kl)

with the Hermite-to-Cartesian transform of the outer-loop side hoisted out
of the inner primitive loop (W/V hold the inner-side-transformed,
inner-primitive-summed Hermite integrals of one outer primitive).  Only
non-zero Hermite coefficients are emitted.

Primitive-pair record fields (SoA, ``base[(f * kmax + k) * stride + pair]``;
the primitive Schwarz factors sit beside them in ``q[k * stride + pair]``):
    0 Px, 1 Py, 2 Pz, 3 p, 4 K (sqrt(2 pi^{5/2}) c_a c_b N_a N_b exp(-mu AB^2) / p),
    5 h = 1/(2p), 6-8 PA = P - A, 9-11 PB = P - B.
ss pairs use fields 0-4, ps pairs 0-8, pp pairs 0-11.
"""
from __future__ import annotations

import itertools
import os

AX = "xyz"
COMPS = {0: [(0, 0, 0)], 1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)]}
# (La, Lb, Lc, Ld, nsplit, loop order); nsplit > 1 splits the c components
# across threads.  'ket' order keeps each thread's ket records in the outer
# loop (read once per quartet, the bra records re-read as warp broadcasts);
# it costs no extra FMAs where the bra and ket transforms are equally cheap.
CLASSES = [
    (0, 0, 0, 0, 1, "ket"),
    (1, 0, 0, 0, 1, "bra"),
    (1, 0, 1, 0, 1, "ket"),
    (1, 1, 0, 0, 1, "bra"),
    (1, 1, 1, 0, 1, "bra"),
    (1, 1, 1, 1, 3, "bra"),
]
PAIR_FIELDS = {0: 5, 1: 9, 2: 12}  # record fields the ERI code loads (the stored records add alpha last)
# classes whose inner primitive loop loads the next primitive pair's record
# one iteration ahead
PREFETCH_CLASSES = {0, 3, 5}  # measured on B200: the others lose more to register spills
# classes whose FP32 instantiation prefetches although the FP64 one does not
# (FP32 records take half the registers; measured on B200, mixed (H2O)_64
# build: (pp|ps) 0.60 -> 0.56 ms, while (ps|ps) loses, 1.28 -> 1.38)
PREFETCH_FP32_CLASSES = {1, 4}
# classes whose outer side's transform fields (h, PA, PB and the Hermite
# coefficients built from them) are loaded after the inner primitive loop,
# where the outer-side Hermite-to-Cartesian transform uses them, so they hold
# no registers across the loop (measured on B200: (ps|ps) 3.29 -> 3.17 ms,
# (pp|ss) 1.79 -> 1.62, (pp|ps) 1.74 -> 1.63 per (H2O)_64 build; (ps|ss)
# 9.0 -> 9.3, so it loads them up front)
DEFER_CLASSES = {2, 3, 4, 5}


def e1d(side, a, b, axis):
    """Non-zero 1-D Hermite coefficients {t: expr} for powers (a, b) on an axis."""
    x = AX[axis]
    if (a, b) == (0, 0):
        return {0: None}
    if (a, b) == (1, 0):
        return {0: f"{side}A{x}", 1: f"{side}h"}
    if (a, b) == (0, 1):
        return {0: f"{side}B{x}", 1: f"{side}h"}
    return {0: f"{side}E{x}0", 1: f"{side}E{x}1", 2: f"{side}h2"}


def e3d(side, ca, cb, sign=False):
    """List of ((t,u,v), sign, factors) for the product of three 1-D expansions."""
    out = []
    per_axis = [e1d(side, ca[k], cb[k], k) for k in range(3)]
    for t, u, v in itertools.product(*[sorted(d) for d in per_axis]):
        facs = [f for f in (per_axis[0][t], per_axis[1][u], per_axis[2][v]) if f is not None]
        sg = -1 if (sign and (t + u + v) % 2) else 1
        out.append(((t, u, v), sg, facs))
    return out


def herm(L):
    return [(t, u, v) for t in range(L + 1) for u in range(L + 1) for v in range(L + 1) if t + u + v <= L]


def rname(t, u, v, n):
    return f"R{t}{u}{v}_{n}"


def r_program(needed, L):
    """Emit R^{(n)}_{tuv} definitions closing `needed` under the MD recursion."""
    need = set()

    def add(t, u, v, n):
        if (t, u, v, n) in need:
            return
        need.add((t, u, v, n))
        if t > 0:
            add(t - 1, u, v, n + 1)
            if t > 1:
                add(t - 2, u, v, n + 1)
        elif u > 0:
            add(t, u - 1, v, n + 1)
            if u > 1:
                add(t, u - 2, v, n + 1)
        elif v > 0:
            add(t, u, v - 1, n + 1)
            if v > 1:
                add(t, u, v - 2, n + 1)

    for t, u, v in needed:
        add(t, u, v, 0)
    lines = []
    base_n = sorted(n for (t, u, v, n) in need if t + u + v == 0)
    maxn = max(base_n)
    lines.append("T cpow = pre;")
    for n in range(maxn + 1):
        if n > 0:
            lines.append("cpow *= m2rho;")
        if n in base_n:
            lines.append(f"const T {rname(0, 0, 0, n)} = cpow * F[{n}];")
    for (t, u, v, n) in sorted(need, key=lambda k: (k[0] + k[1] + k[2], -k[3], k)):
        if t + u + v == 0:
            continue
        if t > 0:
            e = f"X * {rname(t - 1, u, v, n + 1)}"
            if t > 1:
                e += f" + T({t - 1}) * {rname(t - 2, u, v, n + 1)}"
        elif u > 0:
            e = f"Y * {rname(t, u - 1, v, n + 1)}"
            if u > 1:
                e += f" + T({u - 1}) * {rname(t, u - 2, v, n + 1)}"
        else:
            e = f"Z * {rname(t, u, v - 1, n + 1)}"
            if v > 1:
                e += f" + T({v - 1}) * {rname(t, u, v - 2, n + 1)}"
        lines.append(f"const T {rname(t, u, v, n)} = {e};")
    return lines


def prod(facs):
    return " * ".join(facs) if facs else "T(1)"


N_CORE_FIELDS = 5  # Px, Py, Pz, p, K: what the primitive-quartet core reads


def side_loads(side, pc, var, idx, first=0, last=None):
    """Load fields [first, last) of one primitive pair record through the
    per-thread base pointer {var}_p (32-bit offsets: field f at f * {var}_fs);
    the record pointer is declared with the first field range."""
    names = ["Px", "Py", "Pz", "p", "K", "h", "Ax", "Ay", "Az", "Bx", "By", "Bz"]
    n = PAIR_FIELDS[pc] if last is None else min(last, PAIR_FIELDS[pc])
    out = [f"const T* __restrict__ {side}rec = {var}_p + {idx} * {var}_st;"] if first == 0 else []
    for f in range(first, n):
        off = "0" if f == 0 else (f"{var}_fs" if f == 1 else f"{f} * {var}_fs")
        out.append(f"const T {side}{names[f]} = __ldg({side}rec + {off});")
    return out


def side_fields(pc, var):
    """(name, offset expression) of the record fields a pair class reads."""
    names = ["Px", "Py", "Pz", "p", "K", "h", "Ax", "Ay", "Az", "Bx", "By", "Bz"]
    return [(names[f], "0" if f == 0 else (f"{var}_fs" if f == 1 else f"{f} * {var}_fs"))
            for f in range(PAIR_FIELDS[pc])]


def prefetched_inner_loop(side, pc, var, idx, n, qo, other_q):
    """Head of an inner primitive loop whose record fields and primitive
    Schwarz factor are loaded one iteration ahead (software pipelining: the
    loads of primitive j + 1 are in flight while primitive j is computed)."""
    f = side_fields(pc, var)
    q = f"{var}_qp"
    out = [f"float {side}nq = __ldg({q});"]
    out.append("T " + ", ".join(f"{side}n{nm} = __ldg({var}_p + {off})" for nm, off in f) + ";")
    out.append("#pragma unroll 1")
    out.append(f"for (int {idx} = 0; {idx} < {n}; ++{idx}) {{")
    out.append(f"  const float {side}cq = {side}nq;")
    out.append("  const T " + ", ".join(f"{side}{nm} = {side}n{nm}" for nm, _ in f) + ";")
    out.append(f"  if ({qo} * {side}cq < eps) break;")
    out.append(f"  const int {idx}n = {idx} + 1 < {n} ? {idx} + 1 : {idx};")
    out.append(f"  {side}nq = __ldg({q} + {idx}n * {var}_st);")
    out.append(f"  const T* __restrict__ {side}nrec = {var}_p + {idx}n * {var}_st;")
    for nm, off in f:
        out.append(f"  {side}n{nm} = __ldg({side}nrec + {off});")
    return out


CORE_NAMES = ["Px", "Py", "Pz", "p", "K", "qd", "h", "zz"]  # packed core record slots


def core_inner_loop(side, pc, var, idx, n, qo, prefetch):
    """Head of an inner primitive loop that reads each primitive pair's packed
    core record (P, p, K, q, 1/(2p): one 64-byte FP64 or 32-byte FP32 record,
    core_ld) and the remaining transform fields (PA, PB) from the SoA
    records; with `prefetch` the next core record is loaded one iteration
    ahead."""
    names = [f"{side}{nm}" for nm in CORE_NAMES]
    nxt = [f"{side}n{k}" for k in range(8)]
    out = []
    if prefetch:
        out.append("T " + ", ".join(nxt) + ";")
        out.append(f"core_ld({var}_c, {', '.join(nxt)});")
        out.append("#pragma unroll 1")
        out.append(f"for (int {idx} = 0; {idx} < {n}; ++{idx}) {{")
        out.append("  const T " + ", ".join(f"{a} = {b}" for a, b in zip(names, nxt)) + ";")
        out.append(f"  if ({qo} * (float){side}qd < eps) break;")
        out.append(f"  const int {idx}n = {idx} + 1 < {n} ? {idx} + 1 : {idx};")
        out.append(f"  core_ld({var}_c + {idx}n * {var}_cst, {', '.join(nxt)});")
    else:
        out.append("#pragma unroll 1")
        out.append(f"for (int {idx} = 0; {idx} < {n}; ++{idx}) {{")
        out.append("  T " + ", ".join(names) + ";")
        out.append(f"  core_ld({var}_c + {idx} * {var}_cst, {', '.join(names)});")
        out.append(f"  if ({qo} * (float){side}qd < eps) break;")
    extra = {0: [], 1: [6, 7, 8], 2: [6, 7, 8, 9, 10, 11]}[pc]
    if extra:
        fn = ["Px", "Py", "Pz", "p", "K", "h", "Ax", "Ay", "Az", "Bx", "By", "Bz"]
        out.append(f"  const T* __restrict__ {side}rec = {var}_p + {idx} * {var}_st;")
        for f in extra:
            out.append(f"  const T {side}{fn[f]} = __ldg({side}rec + {f} * {var}_fs);")
    return out


def side_pre(side, pc):
    lines = []
    if pc == 2:
        for x in AX:
            lines.append(f"const T {side}E{x}0 = {side}A{x} * {side}B{x} + {side}h;")
            lines.append(f"const T {side}E{x}1 = {side}h * ({side}A{x} + {side}B{x});")
        lines.append(f"const T {side}h2 = {side}h * {side}h;")
    return lines


def inner_loop_variants(cid, side, pc, var, idx, n, qo, inner_pre, inner, uniform):
    """The inner primitive loop (indented into the outer loop's body), FP32
    and FP64 forms behind a switch.  FP32 reads the packed core records; FP64
    reads them where the inner side is the warp-uniform one (`uniform`: two
    broadcast vector loads instead of six) and keeps the SoA fields where
    every lane reads its own pair (64-byte records per lane cost more L1
    wavefronts than five coalesced 8-byte fields: measured on B200, (ps|ss)
    9.1 -> 10.8 ms and (pp|ss) 1.7 -> 2.1 ms per (H2O)_64 build)."""
    q = f"{var}_qp"

    def core_form(pf):
        head = core_inner_loop(side, pc, var, idx, n, qo, pf)
        return head + ["  ++evaluated;"] + ["  " + x for x in inner_pre + inner] + ["}"]

    def soa_form(pf):
        if pf:
            head = prefetched_inner_loop(side, pc, var, idx, n, qo, q)
        else:
            head = ["#pragma unroll 1", f"for (int {idx} = 0; {idx} < {n}; ++{idx}) {{",
                    f"  if ({qo} * __ldg({q} + {idx} * {var}_st) < eps) break;"]
            head += ["  " + x for x in side_loads(side, pc, var, idx)]
        return head + ["  ++evaluated;"] + ["  " + x for x in inner_pre + inner] + ["}"]

    pf32 = cid in PREFETCH_CLASSES or cid in PREFETCH_FP32_CLASSES
    pf64 = cid in PREFETCH_CLASSES
    f64 = core_form(pf64) if uniform else soa_form(pf64)
    lines = ["if constexpr (sizeof(T) == 4) {"] + ["  " + x for x in core_form(pf32)] + ["} else {"]
    lines += ["  " + x for x in f64] + ["}"]
    return ["  " + x for x in lines]


def gen_class(cid, la, lb, lc, ld, nsplit, split, order):
    """order 'bra': bra primitive loop outside, the ket transform per primitive
    quartet and the bra transform hoisted; order 'ket': the mirror image (ket
    records loaded once per quartet, bra records re-read as warp-broadcast)."""
    pa, pk = la + lb, lc + ld
    L = pa + pk
    A, B, C, D = COMPS[la], COMPS[lb], COMPS[lc], COMPS[ld]
    cds = [(ic, id_) for ic in range(len(C)) for id_ in range(len(D))]
    if nsplit > 1:
        cds = [(ic, id_) for (ic, id_) in cds if ic == split]
    abs_ = [(ia, ib) for ia in range(len(A)) for ib in range(len(B))]
    ket_terms = {m: e3d("k", C[ic], D[id_], sign=True) for m, (ic, id_) in enumerate(cds)}
    bra_terms = {n: e3d("b", A[ia], B[ib]) for n, (ia, ib) in enumerate(abs_)}
    hb, hk = herm(pa), herm(pk)
    needed = set()
    for m, terms in ket_terms.items():
        for (tk, uk, vk), _, _ in terms:
            for (tb, ub, vb) in hb:
                needed.add((tb + tk, ub + uk, vb + vk))
    nloc = len(abs_) * len(cds)
    core = [
        "const T s = bp + kp;",
        "const T rs = Math<T>::rsqrt(s);",
        "const T rho = bp * kp * (rs * rs);",
        "const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;",
        "const T pre = bK * kK * rs;",
    ]
    if L > 0:
        core.append("const T m2rho = T(-2) * rho;")
    core.append(f"T F[{L + 1}];")
    core.append(f"Boys<T, {L}>::eval(rho * (X * X + Y * Y + Z * Z), F);")
    core += r_program(sorted(needed), L)
    body = []
    if order == "bra":
        w = lambda m, h: f"W{m}_{h[0]}{h[1]}{h[2]}"
        body.append("const float kq0 = ket_qp[0];")
        body.append("#pragma unroll 1")
        body.append("for (int i = 0; i < bra_n; ++i) {")
        body.append("  const float qo = __ldg(bra_qp + i * bra_st);")
        body.append("  if (qo * kq0 < eps) break;")
        ncore = N_CORE_FIELDS if cid in DEFER_CLASSES else None
        body += ["  " + x for x in side_loads("b", pa, "bra", "i", 0, ncore)]
        for m in range(len(cds)):
            body.append("  T " + ", ".join(f"{w(m, h)} = T(0)" for h in hb) + ";")
        inner_pre = side_pre("k", pk)
        inner = list(core)
        for m, terms in ket_terms.items():
            for (tk, uk, vk), sg, facs in terms:
                cname = f"kc{m}_{tk}{uk}{vk}"
                if facs:
                    inner.append(f"const T {cname} = {'-' if sg < 0 else ''}{prod(facs)};")
                for (tb, ub, vb) in hb:
                    r = rname(tb + tk, ub + uk, vb + vk, 0)
                    tgt = w(m, (tb, ub, vb))
                    if facs:
                        inner.append(f"{tgt} = fma({cname}, {r}, {tgt});")
                    else:
                        inner.append(f"{tgt} {'-=' if sg < 0 else '+='} {r};")
        body += inner_loop_variants(cid, "k", pk, "ket", "j", "ket_n", "qo", inner_pre, inner, False)
        if ncore is not None:
            body += ["  " + x for x in side_loads("b", pa, "bra", "i", ncore)]
        body += ["  " + x for x in side_pre("b", pa)]
        for n, terms in bra_terms.items():
            for m in range(len(cds)):
                acc = f"I[{n * len(cds) + m}]"
                for (tb, ub, vb), _, facs in terms:
                    src = w(m, (tb, ub, vb))
                    body.append(f"  {acc} = fma({prod(facs)}, {src}, {acc});" if facs else f"  {acc} += {src};")
        body.append("}")
    else:
        w = lambda n, h: f"V{n}_{h[0]}{h[1]}{h[2]}"
        body.append("const float bq0 = bra_qp[0];")
        body.append("#pragma unroll 1")
        body.append("for (int j = 0; j < ket_n; ++j) {")
        body.append("  const float qo = __ldg(ket_qp + j * ket_st);")
        body.append("  if (qo * bq0 < eps) break;")
        ncore = N_CORE_FIELDS if cid in DEFER_CLASSES else None
        body += ["  " + x for x in side_loads("k", pk, "ket", "j", 0, ncore)]
        for n in range(len(abs_)):
            body.append("  T " + ", ".join(f"{w(n, h)} = T(0)" for h in hk) + ";")
        inner_pre = side_pre("b", pa)
        inner = list(core)
        for n, terms in bra_terms.items():
            for (tb, ub, vb), _, facs in terms:
                cname = f"bc{n}_{tb}{ub}{vb}"
                if facs:
                    inner.append(f"const T {cname} = {prod(facs)};")
                for (tk, uk, vk) in hk:
                    r = rname(tb + tk, ub + uk, vb + vk, 0)
                    tgt = w(n, (tk, uk, vk))
                    inner.append(f"{tgt} = fma({cname}, {r}, {tgt});" if facs else f"{tgt} += {r};")
        body += inner_loop_variants(cid, "b", pa, "bra", "i", "bra_n", "qo", inner_pre, inner, True)
        if ncore is not None:
            body += ["  " + x for x in side_loads("k", pk, "ket", "j", ncore)]
        body += ["  " + x for x in side_pre("k", pk)]
        # ket transform with the (-1)^{tau+nu+phi} sign
        for m, terms in ket_terms.items():
            for n in range(len(abs_)):
                acc = f"I[{n * len(cds) + m}]"
                for (tk, uk, vk), sg, facs in terms:
                    src = w(n, (tk, uk, vk))
                    if facs:
                        body.append(f"  {acc} = fma({'-' if sg < 0 else ''}{prod(facs)}, {src}, {acc});")
                    else:
                        body.append(f"  {acc} {'-=' if sg < 0 else '+='} {src};")
        body.append("}")
    cd_c = ", ".join(str(ic) for ic, _ in cds)
    cd_d = ", ".join(str(id_) for _, id_ in cds)
    head = [
        f"// class {cid}: ({'sp'[la]}{'sp'[lb]}|{'sp'[lc]}{'sp'[ld]}), split {split} of {nsplit}, {order} primitives outside",
        "template <typename T>",
        f"struct EriClass<T, {cid}, {split}> {{",
        f"  static constexpr int LA = {la}, LB = {lb}, LC = {lc}, LD = {ld}, L = {L};",
        f"  static constexpr int NA = {len(A)}, NB = {len(B)}, NC = {len(C)}, ND = {len(D)};",
        f"  static constexpr int NSPLIT = {nsplit}, NCD = {len(cds)}, NI = {nloc};",
        f"  static constexpr int BRA_CLASS = {pa}, KET_CLASS = {pk};",
        f"  __device__ static constexpr int cd_c(int m) {{ constexpr int v[] = {{{cd_c}}}; return v[m]; }}",
        f"  __device__ static constexpr int cd_d(int m) {{ constexpr int v[] = {{{cd_d}}}; return v[m]; }}",
        "  // Returns the number of primitive quartets evaluated: both sides'",
        "  // primitive pairs come sorted by descending primitive Schwarz factor q,",
        "  // and the loops stop once q_bra * q_ket < eps (each skipped primitive",
        "  // quartet is bounded by that product, Cauchy-Schwarz per primitive pair).",
        "  // bra_core / ket_core: packed core records, core[(k * n_pairs + pair) * 8 + slot].",
        "  __device__ __forceinline__ static int run(",
        "      const T* __restrict__ bra, const T* __restrict__ bra_core, const float* __restrict__ bra_q,",
        "      long long bra_stride, int bra_kmax, int bra_row, int bra_n,",
        "      const T* __restrict__ ket, const T* __restrict__ ket_core, const float* __restrict__ ket_q,",
        "      long long ket_stride, int ket_kmax, int ket_row, int ket_n, float eps, T (&I)[NI]) {",
        "    #pragma unroll",
        "    for (int q = 0; q < NI; ++q) I[q] = T(0);",
        "    int evaluated = 0;",
        "    const int bra_st = (int)bra_stride, ket_st = (int)ket_stride;",
        "    [[maybe_unused]] const int bra_fs = bra_kmax * bra_st, ket_fs = ket_kmax * ket_st;",
        "    const T* __restrict__ bra_p = bra + bra_row;",
        "    const T* __restrict__ ket_p = ket + ket_row;",
        "    const float* __restrict__ bra_qp = bra_q + bra_row;",
        "    const float* __restrict__ ket_qp = ket_q + ket_row;",
        "    const T* __restrict__ bra_c = bra_core + 8 * bra_row;",
        "    const T* __restrict__ ket_c = ket_core + 8 * ket_row;",
        "    [[maybe_unused]] const int bra_cst = 8 * bra_st, ket_cst = 8 * ket_st;",
    ]
    tail = ["    return evaluated;", "  }", "};", ""]
    return head + ["    " + x for x in body] + tail


def main():
    out = [
        "// GENERATED by gen_eri.py -- do not edit by hand.",
        "// Straight-line McMurchie-Davidson bodies for the s/p ERI classes.",
        "#pragma once",
        "",
        "template <typename T, int C, int S> struct EriClass;",
        "",
        f"#define DFTK_N_CLASSES {len(CLASSES)}",
        "",
    ]
    for cid, (la, lb, lc, ld, ns, order) in enumerate(CLASSES):
        for s in range(ns):
            out += gen_class(cid, la, lb, lc, ld, ns, s, order)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "eri_classes.cuh")
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")
    print(path)


if __name__ == "__main__":
    main()
