"""Generates taylor_gen.cuh: straight-line far-field evaluation per Taylor order.

The reference evaluates a particle-cluster interaction (treecode3d_pb.f:439-486
COMPP_TREE_PB) by filling the Taylor-coefficient arrays a(i,j,k), b(i,j,k) of
e^{-kappa r}/r with the recurrences of COMP_TCOEFF (treecode3d_pb.f:684-855)
for kappa = 0 and kappa, then contracting them with 16 weighted cluster moments
(der_cof(k,idx) * ms(idx,k), main.f90:380-399 and treecode3d_pb.f:859-916).

This script emits, for each order P, a device function that
  * computes a(i,j,k) (and b for kappa != 0) only for i+j+k <= P+2 (the
    entries the contraction reads; each entry uses the same recurrence formula
    the reference uses for its index pattern, so its value is the same),
  * walks the entries shell by shell (total degree 0, 1, ...), so that a value
    stays live for at most two further shells and the arrays live in registers,
  * folds every a(m) into the contraction sums as soon as it is known, with
    the moments pre-weighted by the integer part of der_cof (the 16 index
    sums fold into 8 accumulators, one per distinct target charge),
  * drops every b term for kappa = 0 (there b(0,0,0) = 1 is only ever
    multiplied by kappa = 0, and all other b vanish).
Output: the two potentials of COMPP_TREE_PB before the 1/(4 pi) factor.

Usage: python gen_taylor.py [max_order]   (writes taylor_gen.cuh beside itself)
"""
import os
import sys

KK = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0),
      (1, 1, 0), (1, 0, 1), (1, 1, 0), (0, 2, 0), (0, 1, 1), (1, 0, 1), (0, 1, 1), (0, 0, 2)]


# The 16 contraction sums fold into 8 accumulators per kappa: indices with the
# same target charge (pb_kernel, main.f90:671-690) share one: idx 1 (charge 1),
# idx 2-4 (charge 1), idx 5/6/7 (n_x/n_y/n_z), idx 8+3i+j (n_j) for j = x,y,z.
BARRIER = False
ACC_NAMES = ["P", "G", "F0", "F1", "F2", "Hx", "Hy", "Hz"]
ACC_OF = ["P", "G", "G", "G", "F0", "F1", "F2", "Hx", "Hy", "Hz", "Hx", "Hy", "Hz", "Hx", "Hy",
          "Hz"]


def terms(p):
    """multi-indices with |k| <= p, shell order (the moment layout)."""
    out = []
    for n in range(p + 1):
        for k3 in range(n + 1):
            for k2 in range(n - k3 + 1):
                k1 = n - k3 - k2
                out.append((k1, k2, k3))
    return out


def lit(x):
    return repr(float(x))


def formulas(i, j, k, kap):
    """(b_expr, a_expr) for index (i,j,k) as in COMP_TCOEFF; kap=False drops b."""
    A = lambda x, y, z: f"a_{x}_{y}_{z}"
    B = lambda x, y, z: f"b_{x}_{y}_{z}"
    c1 = lambda n: f"cf1n_{n}"
    c2 = lambda n: f"T({lit(1.0 - 0.5 * (1.0 / n))})"
    c3 = lambda n: f"T({lit(1.0 - (1.0 / n))})"
    idx = (i, j, k)
    nz = [v for v in idx if v]
    if idx == (0, 0, 0):
        return ("ex", "ex / dist") if kap else (None, "T(1.0) / dist")
    # single axis
    if len(nz) == 1:
        ax = [i, j, k].index(nz[0])
        d = "xyz"[ax]
        n = nz[0]

        def e(m):
            t = [0, 0, 0]
            t[ax] = m
            return tuple(t)
        if n == 1:
            b = f"kappa{d} * a_0_0_0"
            a = (f"fac * d{d} * (a_0_0_0 + kappa * b_0_0_0)" if kap else f"fac * d{d} * a_0_0_0")
            return (b if kap else None), a
        b = f"{c1(n)} * (d{d} * {A(*e(n-1))} - {A(*e(n-2))})"
        a = f"fac * (dd{d} * {c2(n)} * {A(*e(n-1))} - {c3(n)} * {A(*e(n-2))}"
        a += (f" + {c1(n)} * (d{d} * {B(*e(n-1))} - {B(*e(n-2))}))" if kap else ")")
        return (b if kap else None), a
    ones = [v == 1 for v in idx]
    if len(nz) == 2:
        # patterns with one zero index
        if idx == (1, 1, 0):
            return (("kappax * a_0_1_0" if kap else None),
                    "fac * (dx * a_0_1_0 + ddy * a_1_0_0" + (" + kappax * b_0_1_0)" if kap else ")"))
        if idx == (1, 0, 1):
            return (("kappax * a_0_0_1" if kap else None),
                    "fac * (dx * a_0_0_1 + ddz * a_1_0_0" + (" + kappax * b_0_0_1)" if kap else ")"))
        if idx == (0, 1, 1):
            return (("kappay * a_0_0_1" if kap else None),
                    "fac * (dy * a_0_0_1 + ddz * a_0_1_0" + (" + kappay * b_0_0_1)" if kap else ")"))
        # one index 1, other >= 2 (COMP_TCOEFF :762-781)
        if i == 1 and j == 0:  # (1,0,n)
            n = k
            return ((f"kappax * a_0_0_{n}" if kap else None),
                    f"fac * (dx * a_0_0_{n} + ddz * a_1_0_{n-1} - a_1_0_{n-2}"
                    + (f" + kappax * b_0_0_{n})" if kap else ")"))
        if i == 0 and j == 1:  # (0,1,n)
            n = k
            return ((f"kappay * a_0_0_{n}" if kap else None),
                    f"fac * (dy * a_0_0_{n} + ddz * a_0_1_{n-1} - a_0_1_{n-2}"
                    + (f" + kappay * b_0_0_{n})" if kap else ")"))
        if i == 0 and k == 1:  # (0,n,1)
            n = j
            return ((f"kappaz * a_0_{n}_0" if kap else None),
                    f"fac * (dz * a_0_{n}_0 + ddy * a_0_{n-1}_1 - a_0_{n-2}_1"
                    + (f" + kappaz * b_0_{n}_0)" if kap else ")"))
        if i == 1 and k == 0:  # (1,n,0)
            n = j
            return ((f"kappax * a_0_{n}_0" if kap else None),
                    f"fac * (dx * a_0_{n}_0 + ddy * a_1_{n-1}_0 - a_1_{n-2}_0"
                    + (f" + kappax * b_0_{n}_0)" if kap else ")"))
        if j == 1 and k == 0:  # (n,1,0)
            n = i
            return ((f"kappay * a_{n}_0_0" if kap else None),
                    f"fac * (dy * a_{n}_0_0 + ddx * a_{n-1}_1_0 - a_{n-2}_1_0"
                    + (f" + kappay * b_{n}_0_0)" if kap else ")"))
        if j == 0 and k == 1:  # (n,0,1)
            n = i
            return ((f"kappaz * a_{n}_0_0" if kap else None),
                    f"fac * (dz * a_{n}_0_0 + ddx * a_{n-1}_0_1 - a_{n-2}_0_1"
                    + (f" + kappaz * b_{n}_0_0)" if kap else ")"))
        # both >= 2 (COMP_TCOEFF :784-800)
        if k == 0:
            b = f"{c1(i)} * (dx * a_{i-1}_{j}_0 - a_{i-2}_{j}_0)"
            a = (f"fac * (ddx * {c2(i)} * a_{i-1}_{j}_0 + ddy * a_{i}_{j-1}_0 - {c3(i)} * a_{i-2}_{j}_0"
                 f" - a_{i}_{j-2}_0")
            a += (f" + {c1(i)} * (dx * b_{i-1}_{j}_0 - b_{i-2}_{j}_0))" if kap else ")")
            return (b if kap else None), a
        if j == 0:
            b = f"{c1(i)} * (dx * a_{i-1}_0_{k} - a_{i-2}_0_{k})"
            a = (f"fac * (ddx * {c2(i)} * a_{i-1}_0_{k} + ddz * a_{i}_0_{k-1} - {c3(i)} * a_{i-2}_0_{k}"
                 f" - a_{i}_0_{k-2}")
            a += (f" + {c1(i)} * (dx * b_{i-1}_0_{k} - b_{i-2}_0_{k}))" if kap else ")")
            return (b if kap else None), a
        # i == 0
        b = f"{c1(j)} * (dy * a_0_{j-1}_{k} - a_0_{j-2}_{k})"
        a = (f"fac * (ddy * {c2(j)} * a_0_{j-1}_{k} + ddz * a_0_{j}_{k-1} - {c3(j)} * a_0_{j-2}_{k}"
             f" - a_0_{j}_{k-2}")
        a += (f" + {c1(j)} * (dy * b_0_{j-1}_{k} - b_0_{j-2}_{k}))" if kap else ")")
        return (b if kap else None), a
    # all three nonzero
    if idx == (1, 1, 1):
        return (("kappax * a_0_1_1" if kap else None),
                "fac * (dx * a_0_1_1 + ddy * a_1_0_1 + ddz * a_1_1_0"
                + (" + kappax * b_0_1_1)" if kap else ")"))
    if sum(ones) == 2:
        if i == 1 and j == 1:
            n = k
            return ((f"kappax * a_0_1_{n}" if kap else None),
                    f"fac * (dx * a_0_1_{n} + ddy * a_1_0_{n} + ddz * a_1_1_{n-1} - a_1_1_{n-2}"
                    + (f" + kappax * b_0_1_{n})" if kap else ")"))
        if i == 1 and k == 1:
            n = j
            return ((f"kappax * a_0_{n}_1" if kap else None),
                    f"fac * (dx * a_0_{n}_1 + ddy * a_1_{n-1}_1 + ddz * a_1_{n}_0 - a_1_{n-2}_1"
                    + (f" + kappax * b_0_{n}_1)" if kap else ")"))
        n = i
        return ((f"kappay * a_{n}_0_1" if kap else None),
                f"fac * (dy * a_{n}_0_1 + ddx * a_{n-1}_1_1 + ddz * a_{n}_1_0 - a_{n-2}_1_1"
                + (f" + kappay * b_{n}_0_1)" if kap else ")"))
    if sum(ones) == 1:
        if i == 1:
            return ((f"kappax * a_0_{j}_{k}" if kap else None),
                    f"fac * (dx * a_0_{j}_{k} + ddy * a_1_{j-1}_{k} + ddz * a_1_{j}_{k-1}"
                    f" - a_1_{j-2}_{k} - a_1_{j}_{k-2}" + (f" + kappax * b_0_{j}_{k})" if kap else ")"))
        if j == 1:
            return ((f"kappay * a_{i}_0_{k}" if kap else None),
                    f"fac * (dy * a_{i}_0_{k} + ddx * a_{i-1}_1_{k} + ddz * a_{i}_1_{k-1}"
                    f" - a_{i-2}_1_{k} - a_{i}_1_{k-2}" + (f" + kappay * b_{i}_0_{k})" if kap else ")"))
        return ((f"kappaz * a_{i}_{j}_0" if kap else None),
                f"fac * (dz * a_{i}_{j}_0 + ddx * a_{i-1}_{j}_1 + ddy * a_{i}_{j-1}_1"
                f" - a_{i-2}_{j}_1 - a_{i}_{j-2}_1" + (f" + kappaz * b_{i}_{j}_0)" if kap else ")"))
    # all >= 2 (COMP_TCOEFF :841-853)
    b = f"{c1(i)} * (dx * a_{i-1}_{j}_{k} - a_{i-2}_{j}_{k})"
    a = (f"fac * (ddx * {c2(i)} * a_{i-1}_{j}_{k} + ddy * a_{i}_{j-1}_{k} + ddz * a_{i}_{j}_{k-1}"
         f" - {c3(i)} * a_{i-2}_{j}_{k} - a_{i}_{j-2}_{k} - a_{i}_{j}_{k-2}")
    a += (f" + {c1(i)} * (dx * b_{i-1}_{j}_{k} - b_{i-2}_{j}_{k}))" if kap else ")")
    return (b if kap else None), a


def gen_pass(p, kap, pre):
    """One kappa pass: declarations, recurrence, contraction into acc{pre}_idx."""
    tl = terms(p)
    tindex = {t: n for n, t in enumerate(tl)}
    nt = len(tl)
    out = []
    top = p + 2
    if kap:
        for n in range(2, top + 1):
            out.append(f"    const T cf1n_{n} = T({lit(1.0 / n)}) * kappa;")
        out.append("    const T ex = exp(-kappa * dist);")
    for name in ACC_NAMES:
        out.append(f"    T {pre}{name} = T(0);")
    out.append("    {")
    for n in range(top + 1):
        if n > 0 and BARRIER:
            out.append("    asm volatile(\"\" ::: \"memory\");  // keep moment loads in their shell")
        for k3 in range(n + 1):
            for k2 in range(n - k3 + 1):
                k1 = n - k3 - k2
                bex, aex = formulas(k1, k2, k3, kap)
                if kap and bex is not None:
                    out.append(f"    const T b_{k1}_{k2}_{k3} = {bex};")
                out.append(f"    const T a_{k1}_{k2}_{k3} = {aex};")
                for idx, kk in enumerate(KK):
                    m = (k1 - kk[0], k2 - kk[1], k3 - kk[2])
                    if min(m) < 0 or sum(m) > p:
                        continue
                    acc = pre + ACC_OF[idx]
                    out.append(f"    {acc} = fma(a_{k1}_{k2}_{k3}, Mw[{idx * nt + tindex[m]}], {acc});")
    out.append("    }")
    return out


def gen_order(p):
    """Two passes per order, each its own non-inlined function: kept apart, each
    pass is register-allocated on its own (about 140 registers, no spills, at
    p = 3); inlined together the scheduler interleaves them and spills."""
    nt = len(terms(p))
    L = [f"// ---- order {p}: {nt} moment terms per index, recurrence to degree {p + 2}"]
    for kap, pre, fn in ((False, "u", "far_pass0"), (True, "v", "far_pass1")):
        L += ["template <typename T>",
              f"__device__ __noinline__ TabiFar4<T> {fn}_p{p}(T dx, T dy, T dz, T kappa,",
              "                                             const T* __restrict__ Mw, T n0, T n1, T n2) {",
              "  const T ddx = T(2) * dx, ddy = T(2) * dy, ddz = T(2) * dz;",
              "  T dist = dx * dx + dy * dy + dz * dz;",
              "  const T fac = T(1) / dist;",
              "  dist = sqrt(dist);"]
        if kap:
            L.append("  const T kappax = kappa * dx, kappay = kappa * dy, kappaz = kappa * dz;")
        L += gen_pass(p, kap, pre)
        L += [f"  TabiFar4<T> r;",
              f"  r.P = {pre}P;",
              f"  r.G = {pre}G;",
              f"  r.nF = n0 * {pre}F0 + n1 * {pre}F1 + n2 * {pre}F2;",
              f"  r.nH = n0 * {pre}Hx + n1 * {pre}Hy + n2 * {pre}Hz;",
              "  return r;",
              "}", ""]
    L += ["template <typename T>",
          f"__device__ __forceinline__ void far_eval_p{p}(T dx, T dy, T dz, T kappa, const T* __restrict__ Mw,",
          "                                               T n0, T n1, T n2, T eps, T inv_eps,",
          "                                               T& out1, T& out2) {",
          f"  const TabiFar4<T> c = far_pass0_p{p}<T>(dx, dy, dz, T(0), Mw, n0, n1, n2);",
          f"  const TabiFar4<T> y = far_pass1_p{p}<T>(dx, dy, dz, kappa, Mw, n0, n1, n2);",
          "  // COMPP_TREE_PB :479-485 (before the 1/(4 pi) of der_cof)",
          "  out1 = (c.P - y.P) + (eps * y.G - c.G);",
          "  out2 = -(c.nF - y.nF * inv_eps) + (y.nH - c.nH);",
          "}", ""]
    return L


def main():
    maxp = int(sys.argv[1]) if len(sys.argv) > 1 else 8
    here = os.path.dirname(os.path.abspath(__file__))
    L = ["// GENERATED by gen_taylor.py -- do not edit.",
         "// Far-field particle-cluster evaluation per Taylor order (see gen_taylor.py).",
         "#pragma once",
         f"#define TABI_MAX_ORDER {maxp}", ""]
    # term tables
    for p in range(1, maxp + 1):
        tl = terms(p)
        L.append(f"__device__ __constant__ const signed char tabi_terms_p{p}[{len(tl)}][3] = {{"
                 + ", ".join("{%d,%d,%d}" % t for t in tl) + "};")
    L.append("")
    L.append("__host__ __device__ constexpr int tabi_nterms(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }")
    L.append("")
    L.append("// Per-pass results: P (index 1), G (2-4), n.F (5-7), n.H (8-16).")
    L.append("template <typename T>")
    L.append("struct TabiFar4 {")
    L.append("  T P, G, nF, nH;")
    L.append("};")
    L.append("")
    for p in range(1, maxp + 1):
        L += gen_order(p)
    L.append("template <int P, typename T>")
    L.append("__device__ __forceinline__ void far_eval(T dx, T dy, T dz, T kappa, const T* __restrict__ Mw,")
    L.append("                                         T n0, T n1, T n2, T eps, T inv_eps, T& o1, T& o2) {")
    for p in range(1, maxp + 1):
        kw = "if" if p == 1 else "else if"
        L.append(f"  {kw} constexpr (P == {p}) far_eval_p{p}<T>(dx, dy, dz, kappa, Mw, n0, n1, n2, eps, inv_eps, o1, o2);")
    L.append("}")
    L.append("")
    L.append("template <int P>")
    L.append("__device__ __forceinline__ const signed char (*tabi_terms())[3] {")
    for p in range(1, maxp + 1):
        kw = "if" if p == 1 else "else if"
        L.append(f"  {kw} constexpr (P == {p}) return tabi_terms_p{p};")
    L.append("  else return nullptr;")
    L.append("}")
    with open(os.path.join(here, "taylor_gen.cuh"), "w") as f:
        f.write("\n".join(L) + "\n")


if __name__ == "__main__":
    main()
