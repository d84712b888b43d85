"""Generate straight-line McMurchie-Davidson code for every ERI class with a
d shell and no f shell: (ds|ss), (ds|ps), (ds|pp), (dp|ss), (dp|ps),
(dp|pp), (dd|ss), (dd|ps), (ds|ds), (dp|ds), (dp|dp), (dd|pp), (dd|ds),
(dd|dp), (dd|dd).  Classes with an f shell stay with the warp-per-quartet
kernel (hl.cuh), whose shared scratch holds their larger Hermite sets.

Writes ``hl_classes.cuh`` next to this file; the build (build.py) runs it, so
the ~10 MB of straight-line code stays out of the repository.  The scheme
is the s/p generator's (gen_eri.py) with the bra primitive loop outside: per bra primitive pair i the ket primitives j are
summed into the Hermite-bra, Cartesian-ket intermediate

    W^{cd}_{tuv}(i) = sum_j sum_{tau nu phi} (-1)^{tau+nu+phi} E^{cd}_{tau nu phi}(j) R_{t+tau,u+nu,v+phi}(i, j)

and after the ket loop I[ab][cd] += E^{ab}_{tuv}(i) W^{cd}_{tuv}(i).  The
Hermite coefficients of a d shell come from the recursion of calc_E
(shelled.py:228-294),

    E^{a+1,b}_t = h E^{ab}_{t-1} + PA E^{ab}_t + (t+1) E^{ab}_{t+1}   (b likewise with PB),

emitted once per bra primitive as named temporaries.  Cartesian components
of the d shell follow combinations() (shelled.py:15-23: xx, xy, yy, xz, yz,
zz) and the block is scaled by 1/sqrt(prod (2 l_i - 1)!!) per component
(normal(), shelled.py:95-101) after the loops.

Records are the generic 13-field pair sets of the d path (SoA,
``base[(f * kmax + k) * stride + pair]``; 0 Px, 1 Py, 2 Pz, 3 p, 4 K, 5 h,
6-8 PA, 9-11 PB); each pair's first shell has the larger momentum.
"""
from __future__ import annotations

import itertools
import math
import os

from gen_eri import herm, prod, r_program, rname

AX = "xyz"
COMPS = {
    0: [(0, 0, 0)],
    1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    2: [(2, 0, 0), (1, 1, 0), (0, 2, 0), (1, 0, 1), (0, 1, 1), (0, 0, 2)],
}
# Pair kinds (l_a >= l_b): 0 ss, 1 ps, 2 pp (the lo set), 3 ds, 4 dp, 5 dd
# (the hi set).  A class is (bra kind | ket kind); its code is split into
# chunks of bra components x chunks of ket components, one chunk per thread,
# so the W intermediates and the block fit in registers.
# (La, Lb, Lc, Ld, bra chunks, ket chunks)
CLASSES = [
    (2, 0, 0, 0, 1, 1),   # 0 (ds|ss)
    (2, 0, 1, 0, 1, 1),   # 1 (ds|ps)
    (2, 0, 1, 1, 1, 3),   # 2 (ds|pp)
    (2, 1, 0, 0, 1, 1),   # 3 (dp|ss)
    (2, 1, 1, 0, 1, 3),   # 4 (dp|ps)
    (2, 1, 1, 1, 1, 9),   # 5 (dp|pp)
    (2, 2, 0, 0, 3, 1),   # 6 (dd|ss)
    (2, 2, 1, 0, 3, 3),   # 7 (dd|ps)
    (2, 0, 2, 0, 1, 3),   # 8 (ds|ds)
    (2, 1, 2, 0, 1, 6),   # 9 (dp|ds)
    (2, 1, 2, 1, 1, 18),  # 10 (dp|dp)
    (2, 2, 1, 1, 3, 9),   # 11 (dd|pp)
    (2, 2, 2, 0, 3, 6),   # 12 (dd|ds)
    (2, 2, 2, 1, 6, 9),   # 13 (dd|dp)
    (2, 2, 2, 2, 6, 18),  # 14 (dd|dd)
]
FIELD_NAMES = ["Px", "Py", "Pz", "p", "K", "h", "Ax", "Ay", "Az", "Bx", "By", "Bz"]


def dfact2(n):
    return 1 if n <= 0 else n * dfact2(n - 2)


def cnorm(comp):
    return 1.0 / math.sqrt(math.prod(dfact2(2 * k - 1) for k in comp))


def e_name(side, x, a, b, t):
    return f"{side}E{x}{a}{b}_{t}"


def e1d(side, a, b, axis):
    """Non-zero 1-D Hermite coefficients {t: name or None (= 1)}."""
    x = AX[axis]
    if (a, b) == (0, 0):
        return {0: None}
    if (a, b) == (1, 0):
        return {0: f"{side}A{x}", 1: f"{side}h"}
    if (a, b) == (0, 1):
        return {0: f"{side}B{x}", 1: f"{side}h"}
    return {t: e_name(side, x, a, b, t) for t in range(a + b + 1)}


def e_defs(side, la, lb):
    """Definitions of E^{ab}_t, a <= la, b <= lb, a + b >= 2, per axis (raise a
    from E^{00}, then b)."""
    lines = []
    for axis, x in enumerate(AX):
        table = {(0, 0): {0: "T(1)"}}
        for a in range(la + 1):
            for b in range(lb + 1):
                if (a, b) == (0, 0):
                    continue
                if (a, b) in ((1, 0), (0, 1)):
                    table[(a, b)] = {t: v for t, v in e1d(side, a, b, axis).items()}
                    continue
                src, shift = ((a - 1, b), f"{side}A{x}") if b == 0 else ((a, b - 1), f"{side}B{x}")
                lower = table[src]
                order = a + b
                cur = {}
                for t in range(order + 1):
                    terms = []
                    if t - 1 in lower:
                        terms.append(f"{side}h * {lower[t - 1]}")
                    if t in lower:
                        terms.append(f"{shift} * {lower[t]}")
                    if t + 1 in lower:
                        terms.append(f"T({t + 1}) * {lower[t + 1]}")
                    nm = e_name(side, x, a, b, t)
                    lines.append(f"const T {nm} = {' + '.join(terms)};")
                    cur[t] = nm
                table[(a, b)] = cur
    return lines


def e3d(side, ca, cb, sign=False):
    out = []
    per_axis = [e1d(side, ca[k], cb[k], k) for k in range(3)]
    for t, u, v in itertools.product(*[sorted(d) for d in per_axis]):
        facs = [f for f in (per_axis[0][t], per_axis[1][u], per_axis[2][v]) if f is not None]
        sg = -1 if (sign and (t + u + v) % 2) else 1
        out.append(((t, u, v), sg, facs))
    return out


def loads(side, var, idx, fields):
    out = [f"const T* __restrict__ {side}rec = {var}_p + {idx} * {var}_st;"]
    for f in fields:
        off = "0" if f == 0 else (f"{var}_fs" if f == 1 else f"{f} * {var}_fs")
        out.append(f"const T {side}{FIELD_NAMES[f]} = __ldg({side}rec + {off});")
    return out


def chunks(items, n):
    size = len(items) // n
    assert size * n == len(items)
    return [items[k * size:(k + 1) * size] for k in range(n)]


def kind(l1, l2):
    return {(0, 0): 0, (1, 0): 1, (1, 1): 2, (2, 0): 3, (2, 1): 4, (2, 2): 5}[(l1, l2)]


def gen_class(cid, la, lb, lc, ld, nab_split, ncd_split, split):
    pa, pk = la + lb, lc + ld
    L = pa + pk
    nsplit = nab_split * ncd_split
    A, B, C, D = COMPS[la], COMPS[lb], COMPS[lc], COMPS[ld]
    all_cds = [(ic, id_) for ic in range(len(C)) for id_ in range(len(D))]
    all_abs = [(ia, ib) for ia in range(len(A)) for ib in range(len(B))]
    abs_ = chunks(all_abs, nab_split)[split // ncd_split]
    cds = chunks(all_cds, ncd_split)[split % ncd_split]
    ket_terms = {m: e3d("k", C[ic], D[id_], sign=True) for m, (ic, id_) in enumerate(cds)}
    bra_terms = {n: e3d("b", A[ia], B[ib]) for n, (ia, ib) in enumerate(abs_)}
    # Hermite bra indices this chunk's bra components use
    hb_used = set()
    for terms in bra_terms.values():
        for h, _, _ in terms:
            hb_used.add(h)
    hb = [h for h in herm(pa) if h in hb_used]
    needed = set()
    for terms in ket_terms.values():
        for (tk, uk, vk), _, _ in terms:
            for (tb, ub, vb) in hb:
                needed.add((tb + tk, ub + uk, vb + vk))
    nloc = len(abs_) * len(cds)
    w = lambda m, h: f"W{m}_{h[0]}{h[1]}{h[2]}"
    core = [
        "const T s = bp + kp;",
        "const T rs = Math<T>::rsqrt(s);",
        "const T rho = bp * kp * (rs * rs);",
        "const T X = bPx - kPx, Y = bPy - kPy, Z = bPz - kPz;",
        "const T pre = bK * kK * rs;",
        "const T m2rho = T(-2) * rho;",
        f"T F[{L + 1}];",
        f"Boys<T, {L}>::eval(rho * (X * X + Y * Y + Z * Z), F);",
    ]
    core += r_program(sorted(needed), L)
    body = ["const float kq0 = ket_qp[0];", "#pragma unroll 1", "for (int i = 0; i < bra_n; ++i) {",
            "  const float qo = __ldg(bra_qp + i * bra_st);", "  if (qo * kq0 < eps) break;"]
    body += ["  " + x for x in loads("b", "bra", "i", range(5))]
    for m in range(len(cds)):
        body.append("  T " + ", ".join(f"{w(m, h)} = T(0)" for h in hb) + ";")
    inner = ["#pragma unroll 1", "for (int j = 0; j < ket_n; ++j) {",
             "  if (qo * __ldg(ket_qp + j * ket_st) < eps) break;"]
    nket_fields = 5 if pk == 0 else (9 if ld == 0 else 12)
    inner += ["  " + x for x in loads("k", "ket", "j", range(nket_fields))]
    inner.append("  ++evaluated;")
    if (lc, ld) not in ((0, 0), (1, 0)):
        inner += ["  " + x for x in e_defs("k", lc, ld)]
    inner += ["  " + x for x in core]
    for m, terms in ket_terms.items():
        for (tk, uk, vk), sg, facs in terms:
            cname = f"kc{m}_{tk}{uk}{vk}"
            if facs:
                inner.append(f"  const T {cname} = {'-' if sg < 0 else ''}{prod(facs)};")
            for (tb, ub, vb) in hb:
                r = rname(tb + tk, ub + uk, vb + vk, 0)
                tgt = w(m, (tb, ub, vb))
                if facs:
                    inner.append(f"  {tgt} = fma({cname}, {r}, {tgt});")
                else:
                    inner.append(f"  {tgt} {'-=' if sg < 0 else '+='} {r};")
    inner.append("}")
    body += ["  " + x for x in inner]
    # the bra transform fields, loaded after the ket loop
    body.append("  const T* __restrict__ btrec = bra_p + i * bra_st;")
    for f in range(5, 12):
        body.append(f"  const T b{FIELD_NAMES[f]} = __ldg(btrec + {f} * bra_fs);")
    body += ["  " + x for x in e_defs("b", la, lb)]
    for n, terms in bra_terms.items():
        for m in range(len(cds)):
            acc = f"I[{n * len(cds) + m}]"
            for (tb, ub, vb), _, facs in terms:
                src = w(m, (tb, ub, vb))
                body.append(f"  {acc} = fma({prod(facs)}, {src}, {acc});" if facs else f"  {acc} += {src};")
    body.append("}")
    # component normalisation
    for n, (ia, ib) in enumerate(abs_):
        for m, (ic, id_) in enumerate(cds):
            f = cnorm(A[ia]) * cnorm(B[ib]) * cnorm(C[ic]) * cnorm(D[id_])
            if f != 1.0:
                body.append(f"I[{n * len(cds) + m}] *= T({f!r});")
    cd_c = ", ".join(str(ic) for ic, _ in cds)
    cd_d = ", ".join(str(id_) for _, id_ in cds)
    ab_a = ", ".join(str(ia) for ia, _ in abs_)
    ab_b = ", ".join(str(ib) for _, ib in abs_)
    nm = "spd"
    head = [
        f"// class {cid}: ({nm[la]}{nm[lb]}|{nm[lc]}{nm[ld]}), split {split} of {nsplit}: bra components"
        f" {', '.join(f'{ia}{ib}' for ia, ib in abs_)}, ket components {', '.join(f'{ic}{id_}' for ic, id_ in cds)}",
        "template <typename T>",
        f"struct HlClass<T, {cid}, {split}> {{",
        f"  static constexpr int LA = {la}, LB = {lb}, LC = {lc}, LD = {ld}, L = {L};",
        f"  static constexpr int NA = {len(A)}, NB = {len(B)}, NC = {len(C)}, ND = {len(D)};",
        f"  static constexpr int NSPLIT = {nsplit}, NAB = {len(abs_)}, NCD = {len(cds)}, NI = {nloc};",
        f"  static constexpr int BRA_KIND = {kind(la, lb)}, KET_KIND = {kind(lc, ld)};",
        f"  __device__ static constexpr int ab_a(int n) {{ constexpr int v[] = {{{ab_a}}}; return v[n]; }}",
        f"  __device__ static constexpr int ab_b(int n) {{ constexpr int v[] = {{{ab_b}}}; return v[n]; }}",
        f"  __device__ static constexpr int cd_c(int m) {{ constexpr int v[] = {{{cd_c}}}; return v[m]; }}",
        f"  __device__ static constexpr int cd_d(int m) {{ constexpr int v[] = {{{cd_d}}}; return v[m]; }}",
        "  // Contracted, normalised block I[n NCD + m] (bra component n, ket m) of one quartet;",
        "  // returns the primitive quartets evaluated (both sides sorted by",
        "  // descending primitive Schwarz factor, loops stop once q_bra q_ket < eps).",
        "  __device__ __forceinline__ static int run(",
        "      const T* __restrict__ bra, const float* __restrict__ bra_q, long long bra_stride, int bra_kmax,",
        "      int bra_row, int bra_n, const T* __restrict__ ket, const float* __restrict__ ket_q,",
        "      long long ket_stride, int ket_kmax, int ket_row, int ket_n, float eps, T (&I)[NI]) {",
        "    #pragma unroll",
        "    for (int q = 0; q < NI; ++q) I[q] = T(0);",
        "    int evaluated = 0;",
        "    const int bra_st = (int)bra_stride, ket_st = (int)ket_stride;",
        "    const int bra_fs = bra_kmax * bra_st, ket_fs = ket_kmax * ket_st;",
        "    const T* __restrict__ bra_p = bra + bra_row;",
        "    const T* __restrict__ ket_p = ket + ket_row;",
        "    const float* __restrict__ bra_qp = bra_q + bra_row;",
        "    const float* __restrict__ ket_qp = ket_q + ket_row;",
    ]
    tail = ["    return evaluated;", "  }", "};", ""]
    return head + ["    " + x for x in body] + tail


def render() -> str:
    out = [
        "// GENERATED by gen_hl.py -- do not edit by hand.",
        "// Straight-line McMurchie-Davidson bodies of the ERI classes with a d",
        "// shell and no f shell.",
        "#pragma once",
        "",
        "template <typename T, int C, int S> struct HlClass;",
        "",
        f"#define HLC_N_CLASSES {len(CLASSES)}",
        "// (bra kind, ket kind) per class: 0 ss, 1 ps, 2 pp, 3 ds, 4 dp, 5 dd",
        "static const int hlc_class_kinds[HLC_N_CLASSES][2] = {"
        + ", ".join(f"{{{kind(la, lb)}, {kind(lc, ld)}}}" for la, lb, lc, ld, _, _ in CLASSES) + "};",
        "",
    ]
    for cid, (la, lb, lc, ld, nab, ncd) in enumerate(CLASSES):
        for s in range(nab * ncd):
            out += gen_class(cid, la, lb, lc, ld, nab, ncd, s)
    return "\n".join(out) + "\n"


def main():
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hl_classes.cuh")
    with open(path, "w") as fh:
        fh.write(render())
    print(path)


if __name__ == "__main__":
    main()
