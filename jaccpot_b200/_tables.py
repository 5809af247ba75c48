"""Constant tables for the CUDA kernels, generated at build time.

The only non-trivial constants of the real-basis operators are the per-degree
x<->z swap matrices ``B_U`` (multipole side; the local side uses the
transpose).  They follow Dehnen (2014) eq. 63 for the complex basis and the
no-sqrt2 real conversion ``B_U = Q B_complex^T Q^-1`` exactly as
jaccpot/operators/real_dehnen_q.py:49-143 and :300-380 define them; this module
restates that construction in numpy (float64) and writes
``csrc/generated/bu_tables.h`` as a static ``__constant__`` initialiser, so the
kernels need no run-time upload.

``bu_nonzero`` is the sparsity rule the unrolled kernels rely on to skip the
zero entries at compile time: ``B_U`` keeps the cos class (m >= 0) and the sin
class (m < 0) apart (it preserves parity in y) and inside each class only the
entries whose z-parity matches the source's x-parity survive.  ``generate``
asserts that every entry outside that pattern is exactly zero.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np

MAX_ORDER = 10


def _complex_b(ell: int) -> np.ndarray:
    prev = np.ones((1, 1))
    for n in range(ell):
        nn = n + 1
        w = 2 * nn + 1

        def get(m, l):
            if abs(m) > n or abs(l) > n:
                return 0.0
            return prev[m + n, l + n]

        nxt = np.zeros((w, w))
        for mt in range(-nn, nn + 1):
            for lt in range(-nn, nn + 1):
                if abs(mt) <= n:
                    v = 0.5 * (get(mt, lt - 1) - get(mt, lt + 1))
                elif mt == n + 1:
                    v = 0.5 * (get(n, lt - 1) + get(n, lt + 1) + 2.0 * get(n, lt))
                else:
                    v = 0.5 * (get(-n, lt - 1) + get(-n, lt + 1) - 2.0 * get(-n, lt))
                nxt[mt + nn, lt + nn] = v
        prev = nxt
    return prev


def _q(ell: int) -> np.ndarray:
    w = 2 * ell + 1
    q = np.zeros((w, w), dtype=np.complex128)
    q[ell, ell] = 1.0
    for m in range(1, ell + 1):
        ph = (-1.0) ** m
        q[ell + m, ell + m] = 0.5
        q[ell + m, ell - m] = 0.5 * ph
        q[ell - m, ell + m] = -0.5j
        q[ell - m, ell - m] = 0.5j * ph
    return q


def bu_matrix(ell: int) -> np.ndarray:
    """Real multipole-side swap matrix for degree ``ell`` (float64)."""
    q = _q(ell)
    b = _complex_b(ell)
    return np.real(q @ b.T @ np.linalg.inv(q))


def bu_nonzero(ell: int, i: int, j: int) -> bool:
    """Compile-time sparsity rule of ``B_U`` (row i, column j of degree ell)."""
    mi, mj = i - ell, j - ell
    if (mi >= 0) != (mj >= 0):
        return False
    if mi >= 0:
        return (ell + mi + mj) % 2 == 0
    return (ell + abs(mi) + abs(mj)) % 2 == 1


def bu_offset(ell: int) -> int:
    return sum((2 * l + 1) ** 2 for l in range(ell))


def generate(out_path: Path, max_order: int = MAX_ORDER) -> Path:
    vals = []
    for ell in range(max_order + 1):
        b = bu_matrix(ell)
        w = 2 * ell + 1
        for i in range(w):
            for j in range(w):
                if not bu_nonzero(ell, i, j):
                    if b[i, j] != 0.0 and abs(b[i, j]) > 1e-12:
                        raise AssertionError(f"B_U sparsity rule broken at l={ell} ({i},{j})")
                    b[i, j] = 0.0
        vals.extend(b.reshape(-1).tolist())
    lines = [
        "// Generated by jaccpot_b200/_tables.py -- do not edit.",
        "// B_U per degree l (row-major (2l+1)^2), offset sum_{k<l} (2k+1)^2.",
        "#pragma once",
        f"#define JB_BU_MAX_ORDER {max_order}",
        f"static __constant__ float c_BU[{len(vals)}] = {{",
    ]
    for k in range(0, len(vals), 6):
        lines.append("  " + ", ".join(f"{float(np.float32(v))!r}f" for v in vals[k : k + 6]) + ",")
    lines.append("};")
    text = "\n".join(lines) + "\n"
    out_path.parent.mkdir(parents=True, exist_ok=True)
    if not out_path.exists() or out_path.read_text() != text:
        out_path.write_text(text)
    return out_path


def zm2l_matrix(p: int) -> np.ndarray:
    """z-axis M2L in scaled form (operators/real_translations.py:213-335):
    F_n^m r^(n+1) = sum_{k=|m|}^{p-n} sgn(m) (n+k)! (M_k^m r^-k), with
    sgn(m) = (-1)^m (2 if m != 0 else 1); packed indices n^2 + n + m."""
    from math import factorial

    C = (p + 1) ** 2
    z = np.zeros((C, C))
    for n in range(p + 1):
        for m in range(-n, n + 1):
            am = abs(m)
            sg = (-1.0) ** am * (2.0 if m else 1.0)
            for k in range(am, p - n + 1):
                z[n * n + n + m, k * k + k + m] = sg * factorial(n + k)
    return z


def kfold_matrix(p: int) -> np.ndarray:
    """K = B^T Z0 B over all degrees <= p (B block-diagonal per degree).

    B and the degree scalings r^-k / r^-(n+1) commute (B maps each degree to
    itself), so the middle of the rotate+scale chain
    B^T (r^-(n+1) Z0 r^-k) B equals r^-(n+1) K r^-k with K constant."""
    C = (p + 1) ** 2
    b = np.zeros((C, C))
    for ell in range(p + 1):
        b[ell * ell:(ell + 1) ** 2, ell * ell:(ell + 1) ** 2] = bu_matrix(ell)
    k = b.T @ zm2l_matrix(p) @ b
    k[np.abs(k) < 1e-9 * max(1.0, np.abs(k).max())] = 0.0
    return k


def kfold_blocks(k: np.ndarray) -> list[list[int]]:
    """Index sets of the diagonal blocks of K (rows == columns), plus the
    indices that K maps to zero (returned as the last entry)."""
    C = k.shape[0]
    nz = k != 0
    parent = list(range(C))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for i, j in zip(*np.nonzero(nz)):
        parent[find(int(i))] = find(int(j))
    groups: dict[int, list[int]] = {}
    used = nz.any(axis=0) | nz.any(axis=1)
    for i in range(C):
        if used[i]:
            groups.setdefault(find(i), []).append(i)
    blocks = sorted(groups.values(), key=lambda g: (-len(g), g[0]))
    for g in blocks:
        sub = np.zeros(C, dtype=bool)
        sub[g] = True
        assert not (nz[sub][:, ~sub].any() or nz[~sub][:, sub].any()), "K blocks are not square"
    unused = [i for i in range(C) if not used[i]]
    return blocks + [unused]


def _flit(x: float) -> str:
    v = float(np.float32(x))
    return f"{v!r}f" if v != 0 else "0.0f"


def generate_kfold(out_path: Path, max_order: int = MAX_ORDER) -> Path:
    """Unrolled in-place K application per order, K entries as literals."""
    lines = [
        "// Generated by jaccpot_b200/_tables.py -- do not edit.",
        "// In-place v <- K v with K = B^T Z0 B (the constant middle of the real",
        "// rotate+scale M2L), block by block; indices K maps to zero are cleared.",
        "#pragma once",
        "namespace jb {",
        "template <int P> struct KFold;",
    ]
    for p in range(1, max_order + 1):
        k = kfold_matrix(p)
        *blocks, unused = kfold_blocks(k)
        lines.append(f"template <> struct KFold<{p}> {{")
        lines.append(f"  static constexpr int kNnz = {int((k != 0).sum())};")
        lines.append("  static __device__ __forceinline__ void apply(float* v) {")
        for g in blocks:
            lines.append("    {")
            lines.append("      " + " ".join(f"const float i{j} = v[{j}];" for j in g))
            for i in g:
                terms = [(j, k[i, j]) for j in g if k[i, j] != 0]
                expr = f"{_flit(terms[0][1])} * i{terms[0][0]}"
                for j, val in terms[1:]:
                    expr = f"fmaf({_flit(val)}, i{j}, {expr})"
                lines.append(f"      v[{i}] = {expr};")
            lines.append("    }")
        if unused:
            lines.append("    " + " ".join(f"v[{i}] = 0.f;" for i in unused))
        lines.append("  }")
        lines.append("};")
    lines.append("}  // namespace jb")
    text = "\n".join(lines) + "\n"
    out_path.parent.mkdir(parents=True, exist_ok=True)
    if not out_path.exists() or out_path.read_text() != text:
        out_path.write_text(text)
    return out_path


def generate_bu_code(out_path: Path, max_order: int = MAX_ORDER) -> Path:
    """Unrolled v <- B v and v <- B^T v per order with the non-zero B_U entries
    as literals (no constant-memory reads), degree by degree in place."""
    lines = [
        "// Generated by jaccpot_b200/_tables.py -- do not edit.",
        "// In-place v <- B v (TR = false) or B^T v (TR = true) over degrees 1..P,",
        "// B = B_U per degree (its non-zero entries as literals).",
        "#pragma once",
        "namespace jb {",
        "template <int P, bool TR> struct BApply;",
    ]
    for p in range(1, max_order + 1):
        for tr in (False, True):
            lines.append(f"template <> struct BApply<{p}, {'true' if tr else 'false'}> {{")
            lines.append("  static __device__ __forceinline__ void apply(float* v) {")
            for ell in range(1, p + 1):
                b = bu_matrix(ell)
                if tr:
                    b = b.T
                w = 2 * ell + 1
                o = ell * ell
                lines.append("    {")
                lines.append("      " + " ".join(f"const float i{j} = v[{o + j}];" for j in range(w)))
                for i in range(w):
                    terms = [(j, b[i, j]) for j in range(w) if abs(b[i, j]) > 1e-12]
                    if not terms:
                        lines.append(f"      v[{o + i}] = 0.f;")
                        continue
                    expr = f"{_flit(terms[0][1])} * i{terms[0][0]}"
                    for j, val in terms[1:]:
                        expr = f"fmaf({_flit(val)}, i{j}, {expr})"
                    lines.append(f"      v[{o + i}] = {expr};")
                lines.append("    }")
            lines.append("  }")
            lines.append("};")
    # the same blocks one degree at a time (the level kernels split the
    # degrees of one translation over several warps)
    lines.append("template <int L, bool TR> struct BDeg;")
    for ell in range(0, max_order + 1):
        for tr in (False, True):
            lines.append(f"template <> struct BDeg<{ell}, {'true' if tr else 'false'}> {{")
            lines.append("  static __device__ __forceinline__ void apply(float* v) {")
            if ell > 0:
                b = bu_matrix(ell)
                if tr:
                    b = b.T
                w = 2 * ell + 1
                o = ell * ell
                lines.append("    " + " ".join(f"const float i{j} = v[{o + j}];" for j in range(w)))
                for i in range(w):
                    terms = [(j, b[i, j]) for j in range(w) if abs(b[i, j]) > 1e-12]
                    if not terms:
                        lines.append(f"    v[{o + i}] = 0.f;")
                        continue
                    expr = f"{_flit(terms[0][1])} * i{terms[0][0]}"
                    for j, val in terms[1:]:
                        expr = f"fmaf({_flit(val)}, i{j}, {expr})"
                    lines.append(f"    v[{o + i}] = {expr};")
            else:
                lines.append("    (void)v;")
            lines.append("  }")
            lines.append("};")
    lines.append("}  // namespace jb")
    text = "\n".join(lines) + "\n"
    out_path.parent.mkdir(parents=True, exist_ok=True)
    if not out_path.exists() or out_path.read_text() != text:
        out_path.write_text(text)
    return out_path


# ---------------------------------------------------------------------------
# tcgen05 plans for the split-BF16 M2L chain
# ---------------------------------------------------------------------------
TC_ORDERS = tuple(range(2, 9))
TC_ROW = 96  # padded width of the A operand rows (bf16 elements)


def _components(mat: np.ndarray) -> list[tuple[list[int], list[int]]]:
    """Connected components of the bipartite non-zero graph: (rows, cols)."""
    R, Cc = mat.shape
    parent = list(range(R + Cc))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for i, j in zip(*np.nonzero(mat)):
        parent[find(int(i))] = find(R + int(j))
    groups: dict[int, tuple[list[int], list[int]]] = {}
    for i in range(R):
        if mat[i].any():
            groups.setdefault(find(i), ([], []))[0].append(i)
    for j in range(Cc):
        if mat[:, j].any():
            groups.setdefault(find(R + j), ([], []))[1].append(j)
    return list(groups.values())


def _bf16_bits(x: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def _bf16_val(bits: np.ndarray) -> np.ndarray:
    return (bits.astype(np.uint32) << 16).view(np.float32)


def tc_plan(p: int) -> dict:
    """Block-diagonal tensor-core tiling of the three constant products of the
    M2L chain (B, K = B^T Z0 B, B^T) at order p.

    Each product's non-zero structure splits into small square blocks (B: per
    degree, cos / sin class and m-parity; K: four blocks).  Blocks are packed
    first-fit into 16-wide tiles (wider blocks get their own tile, rounded up
    to 16); tile j owns padded columns [col0, col0 + w) of both the input (A
    operand) and the output (TMEM accumulator) index spaces.  `inp[c]` /
    `out[c]` give the coefficient held by padded column c (-1 = zero pad).
    Weights are split into BF16 hi and lo parts, stored per tile as w x w
    K-major core-matrix blocks (8 rows x 16 bytes each)."""
    C = (p + 1) ** 2
    bfull = np.zeros((C, C))
    for ell in range(p + 1):
        bfull[ell * ell:(ell + 1) ** 2, ell * ell:(ell + 1) ** 2] = bu_matrix(ell)
    bfull[np.abs(bfull) < 1e-12] = 0.0
    k = kfold_matrix(p)
    gemms = []
    for mat, pack in ((bfull, True), (k, False), (bfull.T.copy(), True)):
        comps = _components(mat)
        for r, q in comps:
            assert len(r) == len(q), "blocks must be square"
        comps.sort(key=lambda rq: (-len(rq[0]), rq[0][0]))
        bins: list[list] = []
        for r, q in comps:
            w = len(r)
            if pack and w <= 16:
                for b in bins:
                    if b[0] == 16 and b[1] + w <= 16:
                        b[2].append((r, q))
                        b[1] += w
                        break
                else:
                    bins.append([16, w, [(r, q)]])
            else:
                bins.append([(w + 15) // 16 * 16, w, [(r, q)]])
        tiles, inp, out, wbits = [], [], [], []
        col0 = 0
        woff = 0
        for wd, _, blocks in bins:
            rows = [i for r, _ in blocks for i in r]
            cols = [j for _, q in blocks for j in q]
            tile = np.zeros((wd, wd))
            ro, co = 0, 0
            for r, q in blocks:
                tile[ro:ro + len(r), co:co + len(q)] = mat[np.ix_(r, q)]
                ro += len(r)
                co += len(q)
            inp += cols + [-1] * (wd - len(cols))
            out += rows + [-1] * (wd - len(rows))
            hi = _bf16_bits(tile.astype(np.float32))
            lo = _bf16_bits((tile - _bf16_val(hi).astype(np.float64)).astype(np.float32))
            for part in (hi, lo):
                buf = np.zeros(wd * wd, np.uint16)
                for n in range(wd):
                    for kk in range(wd):
                        off = (n // 8) * (wd // 8) * 64 + (kk // 8) * 64 + (n % 8) * 8 + (kk % 8)
                        buf[off] = part[n, kk]
                wbits.append(buf)
            tiles.append((col0, wd, woff))
            col0 += wd
            woff += 2 * wd * wd * 2
        assert col0 <= TC_ROW, (p, col0)
        gemms.append({"tiles": tiles, "inp": inp, "out": out, "npad": col0,
                      "w": np.concatenate(wbits) if wbits else np.zeros(0, np.uint16)})
    return {"p": p, "gemms": gemms}


def generate_tc(out_path: Path) -> Path:
    lines = [
        "// Generated by jaccpot_b200/_tables.py -- do not edit.",
        "// tcgen05 plans of the split-BF16 M2L chain (B, K = B^T Z0 B, B^T) per order:",
        "// tiles (col0, width, byte offset of the hi part; lo follows), padded-column",
        "// to coefficient maps, and the BF16 hi/lo weight tiles in K-major core-matrix",
        "// layout.",
        "#pragma once",
        "#include <stdint.h>",
        "namespace jb {",
        f"constexpr int kTcRow = {TC_ROW};",
        "template <int P> struct TcPlan;",
    ]
    for p in TC_ORDERS:
        pl = tc_plan(p)
        g = pl["gemms"]
        wall = np.concatenate([x["w"] for x in g])
        goff = np.cumsum([0] + [x["w"].size * 2 for x in g])
        lines.append(f"static __device__ __align__(16) const uint16_t c_tc_w_p{p}[{max(wall.size, 1)}] = {{")
        for a in range(0, wall.size, 16):
            lines.append("  " + ", ".join(str(int(v)) for v in wall[a:a + 16]) + ",")
        lines.append("};")
        lines.append(f"template <> struct TcPlan<{p}> {{")
        lines.append(f"  static constexpr int kWBytes = {int(goff[-1])};")
        lines.append(f"  static __device__ __forceinline__ const uint16_t* weights() {{ return c_tc_w_p{p}; }}")
        for gi, x in enumerate(g):
            lines.append(f"  static constexpr int kNumTiles{gi} = {len(x['tiles'])};")
            lines.append(f"  static constexpr int kNpad{gi} = {x['npad']};")
            lines.append(f"  static constexpr int kGemmOff{gi} = {int(goff[gi])};")
            t = x["tiles"]
            lines.append(f"  static __host__ __device__ constexpr int tile_col{gi}(int j) {{ constexpr int t[] = {{{', '.join(str(a) for a, _, _ in t)}}}; return t[j]; }}")
            lines.append(f"  static __host__ __device__ constexpr int tile_w{gi}(int j) {{ constexpr int t[] = {{{', '.join(str(b) for _, b, _ in t)}}}; return t[j]; }}")
            lines.append(f"  static __host__ __device__ constexpr int tile_off{gi}(int j) {{ constexpr int t[] = {{{', '.join(str(int(goff[gi]) + c) for _, _, c in t)}}}; return t[j]; }}")
            lines.append(f"  static __host__ __device__ constexpr int inp{gi}(int c) {{ constexpr int t[] = {{{', '.join(str(v) for v in x['inp'])}}}; return c < {x['npad']} ? t[c] : -1; }}")
            lines.append(f"  static __host__ __device__ constexpr int out{gi}(int c) {{ constexpr int t[] = {{{', '.join(str(v) for v in x['out'])}}}; return c < {x['npad']} ? t[c] : -1; }}")
        lines.append("};")
    lines.append("}  // namespace jb")
    text = "\n".join(lines) + "\n"
    out_path.parent.mkdir(parents=True, exist_ok=True)
    if not out_path.exists() or out_path.read_text() != text:
        out_path.write_text(text)
    return out_path


if __name__ == "__main__":
    generate(Path(__file__).resolve().parent / "csrc" / "generated" / "bu_tables.h")
    generate_tc(Path(__file__).resolve().parent / "csrc" / "generated" / "tc_plans.h")
    generate_bu_code(Path(__file__).resolve().parent / "csrc" / "generated" / "bu_code.h")
    generate_kfold(Path(__file__).resolve().parent / "csrc" / "generated" / "kfold_tables.h")
