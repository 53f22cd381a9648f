"""CPU access to the plan builder of adtlert_b200 and a NumPy replay of its device schedule.

``compile_shim`` builds ``tests/native/host_plan_shim.cpp`` together with the library's own
``plan_host.cpp`` (no CUDA); ``HostPlan`` exposes the tables; the ``replay_*`` functions execute
the solver and assembly tables exactly as the CUDA kernels index them (same offsets, same block
shapes), asserting that every access stays inside its buffer.
"""

from __future__ import annotations

import ctypes
import subprocess
import types
from pathlib import Path

import numpy as np
import scipy.linalg as sla

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "ad-tlert_b200" / "csrc"
BUILD = ROOT / "tests" / "_build"

(T_J, T_MJ, T_OFFJ, T_LOFF, T_P, T_MP, T_OFFP, T_UOFF, T_LINKP, T_Q, T_MQ, T_OFFQ, T_VOFF, T_LINKQ, T_FILL, T_PULL0,
 T_PULL1, T_RUOFF, T_RVOFF) = range(19)
T_FIELDS = 19
P_TYPE, P_OFF, P_ME, P_EOFF, P_AOFF = range(5)

_TYPES = {
    "task_rows": np.int64, "pulls": np.int64, "features": np.float32, "fscale": np.float32,
    "rcv_w": np.float64, "rdof_w": np.float64, "k2": np.float64,
}


def compile_shim() -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    target = BUILD / "libhostplan.so"
    sources = [ROOT / "tests" / "native" / "host_plan_shim.cpp", CSRC / "plan_host.cpp"]
    stale = not target.exists() or any(s.stat().st_mtime > target.stat().st_mtime for s in sources + [CSRC / "plan_host.h"])
    if stale:
        subprocess.run(
            ["g++", "-std=c++17", "-O2", "-shared", "-fPIC", f"-I{ROOT / 'include'}", f"-I{CSRC}", *map(str, sources), "-o", str(target)],
            check=True,
        )
    return target


class HostPlan:
    def __init__(self, problem_struct):
        lib = ctypes.CDLL(str(compile_shim()))
        lib.shim_build.restype = ctypes.c_void_p
        lib.shim_build.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        lib.shim_error.restype = ctypes.c_char_p
        lib.shim_error.argtypes = [ctypes.c_void_p]
        lib.shim_free.argtypes = [ctypes.c_void_p]
        lib.shim_scalar.restype = ctypes.c_longlong
        lib.shim_scalar.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        lib.shim_table.restype = ctypes.c_longlong
        lib.shim_table.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
        status = ctypes.c_int()
        handle = lib.shim_build(ctypes.byref(problem_struct), ctypes.byref(status))
        self.status = status.value
        self.error = lib.shim_error(handle).decode()
        self._lib, self._h = lib, handle
        if self.status == 0:
            for name in ("N", "nnz", "nb", "max_m", "levels", "RS", "R", "rdofs", "factor_stride", "contributions",
                         "tiled"):
                setattr(self, name, int(lib.shim_scalar(handle, name.encode())))
            for name in ("perm", "iperm", "level_begin", "csr_ptr", "csr_col", "csr_row", "contrib_ptr", "contrib",
                         "task_rows", "pulls", "features", "fscale", "pair_ptr", "pair_list", "rcv_dofs", "rcv_w",
                         "rdof_ptr", "rdof_rcv", "rdof_dof", "rdof_w", "cdofs", "bd", "cell_bptr", "cell_blist",
                         "model_ptr", "model_list", "k2", "bowners", "fixed", "titems", "tranges", "panel_ptr",
                         "update_items", "update_begin"):
                size = lib.shim_table(handle, name.encode(), None)
                out = np.empty(size, dtype=_TYPES.get(name, np.int32))
                lib.shim_table(handle, name.encode(), out.ctypes.data_as(ctypes.c_void_p))
                setattr(self, name, out)
            self.tasks = self.task_rows.reshape(-1, T_FIELDS)
            self.pull_table = self.pulls.reshape(-1, 5)

    def __del__(self):
        try:
            self._lib.shim_free(self._h)
        except Exception:
            pass


def replay_assembly(hp: HostPlan, sigma, stiffness, mass, bmass, bcoef, bcells, k2_w, robin=True,
                    identity=True) -> np.ndarray:
    """CSR values of one system as assemble_kernel computes them (solver order)."""

    C, K2 = stiffness.shape[0], stiffness.shape[1] * stiffness.shape[2]
    BL2 = bmass.shape[1] * bmass.shape[2] if bmass.size else 1
    s_flat, m_flat, b_flat = stiffness.reshape(-1), mass.reshape(-1), bmass.reshape(-1)
    out = np.zeros(hp.nnz)
    for slot in range(hp.nnz):
        acc = 0.0
        for code in hp.contrib[hp.contrib_ptr[slot]:hp.contrib_ptr[slot + 1]]:
            if code < 0:
                acc += 1.0 if identity else 0.0
            elif code < C * K2:
                acc += sigma[code // K2] * (s_flat[code] + k2_w * m_flat[code])
            elif robin:
                bc = code - C * K2
                b = bc // BL2
                acc += sigma[bcells[b]] * bcoef[b] * b_flat[bc]
        out[slot] = acc
    return out


def _check(offset, size, stride, what):
    assert 0 <= offset and offset + size <= stride, f"{what}: [{offset}, {offset + size}) outside [0, {stride})"


def _update_items(hp: HostPlan, level: int):
    items = hp.update_items.reshape(-1, 3)
    return items[hp.update_begin[level]:hp.update_begin[level + 1]]


def replay_factor(hp: HostPlan, values: np.ndarray, rhs: np.ndarray | None = None):
    """Factor storage of one system as the shared-memory kernels write it: D of every block
    scattered into its G storage; per level the eliminations (inverse launch: G_j = D_j^-1,
    Z_p = G_j A[j,p], V_q = A[q,j] G_j, coupling copies, fill -A[q,j] Z_p) and the eager Schur
    updates of the neighbouring blocks (A[e,j]^T Z_j, V_j A[j,e]^T). Every access is
    bounds-checked, every read must follow a write, and no item of a launch may write what another
    item of that launch reads or writes. With ``rhs`` (N, nrhs) the update launches also apply the
    forward substitution (b_j -= Z_j^T b_e / V_j b_e, update_rhs_level_kernel) and the forward-
    reduced right-hand side is returned with the factors; its rows join the race checks (indices
    offset past the factor storage)."""

    stride = hp.factor_stride
    x = None if rhs is None else rhs.astype(float).copy()

    def rows(off, count):
        assert 0 <= off and off + count <= x.shape[0], "rhs rows out of range"
        return stride + (np.arange(off, off + count)[:, None] * x.shape[1] + np.arange(x.shape[1])[None, :])
    f = np.full(stride, np.nan)

    def idx(offset, rows, cols, what):
        _check(offset, rows * cols, stride, what)
        return np.arange(offset, offset + rows * cols)

    def load(offset, rows, cols, what):
        block = f[idx(offset, rows, cols, what)].reshape(rows, cols)
        assert np.all(np.isfinite(block)), f"{what}: read before written"
        return block.copy()

    for t in range(len(hp.tasks)):  # scatter launch
        row = hp.tasks[t]
        mj, offj = int(row[T_MJ]), int(row[T_OFFJ])
        dm = np.zeros((mj, mj))
        for s in range(hp.csr_ptr[offj], hp.csr_ptr[offj + mj]):
            c = hp.csr_col[s]
            if offj <= c < offj + mj:
                dm[hp.csr_row[s] - offj, c - offj] = values[s]
        f[idx(int(row[T_LOFF]), mj, mj, "D")] = dm.reshape(-1)
    for level in range(hp.levels):
        launch, results = _Launch("invert"), []
        for t in range(hp.level_begin[level], hp.level_begin[level + 1]):
            row = hp.tasks[t]
            mj, offj = int(row[T_MJ]), int(row[T_OFFJ])
            p, mp, offp = int(row[T_P]), int(row[T_MP]), int(row[T_OFFP])
            q, mq, offq = int(row[T_Q]), int(row[T_MQ]), int(row[T_OFFQ])
            assert 0 < mj <= 64 and (p < 0 or 0 < mp <= 64) and (q < 0 or 0 < mq <= 64)
            p_csr, q_csr = p >= 0 and row[T_LINKP] < 0, q >= 0 and row[T_LINKQ] < 0
            reads = [idx(int(row[T_LOFF]), mj, mj, "D")]
            dm = load(int(row[T_LOFF]), mj, mj, "D")
            ap, aq = np.zeros((mj, max(mp, 0))), np.zeros((max(mq, 0), mj))
            for s in range(hp.csr_ptr[offj], hp.csr_ptr[offj + mj]):
                r, c = hp.csr_row[s] - offj, hp.csr_col[s]
                assert 0 <= r < mj
                if p_csr and offp <= c < offp + mp:
                    ap[r, c - offp] = values[s]
                elif q_csr and offq <= c < offq + mq:
                    aq[c - offq, r] = values[s]
            if p >= 0 and not p_csr:
                ap = load(int(row[T_LINKP]), mj, mp, "link p")
                reads.append(idx(int(row[T_LINKP]), mj, mp, "link p"))
            if q >= 0 and not q_csr:
                aq = load(int(row[T_LINKQ]), mq, mj, "link q")
                reads.append(idx(int(row[T_LINKQ]), mq, mj, "link q"))
            G = np.linalg.inv(dm)
            out = [(int(row[T_LOFF]), G, "G")]
            if p >= 0:
                Z = G @ ap
                out += [(int(row[T_UOFF]), Z, "Z"), (int(row[T_RUOFF]), ap, "coupling p")]
            if q >= 0:
                V = aq @ G
                out += [(int(row[T_VOFF]), V, "V"), (int(row[T_RVOFF]), aq, "coupling q")]
            if p >= 0 and q >= 0:
                out.append((int(row[T_FILL]), -aq @ Z, "fill"))
            launch.item(reads, [idx(off, *block.shape, what) for off, block, what in out])
            results += out
        launch.check()
        for off, block, what in results:
            f[idx(off, *block.shape, what)] = block.reshape(-1)
        launch, results = _Launch("update"), []
        for t, u0, u1 in _update_items(hp, level):
            row = hp.tasks[t]
            mj, loff, offj = int(row[T_MJ]), int(row[T_LOFF]), int(row[T_OFFJ])
            dm = load(loff, mj, mj, "D (update)")
            reads, writes = [idx(loff, mj, mj, "D")], [idx(loff, mj, mj, "D")]
            bj = None
            if x is not None:
                bj = x[offj:offj + mj].copy()
                reads.append(rows(offj, mj))
                writes.append(rows(offj, mj))
            for u in range(u0, u1):
                assert row[T_PULL0] <= u < row[T_PULL1]
                kind, off, me, eoff, aoff = (int(v) for v in hp.pull_table[u])
                if kind == 0:
                    A, Z = load(aoff, me, mj, "coupling"), load(off, me, mj, "Z")
                    dm -= A.T @ Z
                    reads += [idx(aoff, me, mj, "coupling"), idx(off, me, mj, "Z")]
                    if x is not None:
                        bj -= Z.T @ x[eoff:eoff + me]
                else:
                    V, A = load(off, mj, me, "V"), load(aoff, mj, me, "coupling")
                    dm -= V @ A.T
                    reads += [idx(off, mj, me, "V"), idx(aoff, mj, me, "coupling")]
                    if x is not None:
                        bj -= V @ x[eoff:eoff + me]
                if x is not None:
                    reads.append(rows(eoff, me))
            launch.item(reads, writes)
            results.append((loff, dm, offj, bj))
        launch.check()
        for loff, dm, offj, bj in results:
            f[loff:loff + dm.size] = dm.reshape(-1)
            if bj is not None:
                x[offj:offj + bj.shape[0]] = bj
    return f if x is None else (f, x)


def replay_solve(hp: HostPlan, f: np.ndarray, rhs: np.ndarray) -> np.ndarray:
    """Solution of one system for rhs (N, nrhs) in solver order, as the shared-memory kernels
    compute it: forward = the eager updates b_j -= Z_j^T b_e / V_j b_e level by level; backward
    = x_j = G_j b_j - Z_p x_p - V_q^T x_q from the root down."""

    x = rhs.astype(float).copy()

    def block(off, rows, cols):
        return f[off:off + rows * cols].reshape(rows, cols)

    for level in range(hp.levels):
        for t, u0, u1 in _update_items(hp, level):
            row = hp.tasks[t]
            mj, offj = int(row[T_MJ]), int(row[T_OFFJ])
            for u in range(u0, u1):
                kind, off, me, eoff, _ = (int(v) for v in hp.pull_table[u])
                y = x[eoff:eoff + me]
                x[offj:offj + mj] -= (block(off, me, mj).T @ y) if kind == 0 else (block(off, mj, me) @ y)
    return replay_backward(hp, f, x)


def replay_backward(hp: HostPlan, f: np.ndarray, reduced: np.ndarray) -> np.ndarray:
    """The backward levels alone on a forward-reduced right-hand side (backward_level_kernel)."""

    x = reduced.astype(float).copy()

    def block(off, rows, cols):
        return f[off:off + rows * cols].reshape(rows, cols)

    for level in range(hp.levels - 1, -1, -1):
        for t in range(hp.level_begin[level], hp.level_begin[level + 1]):
            row = hp.tasks[t]
            mj, offj = int(row[T_MJ]), int(row[T_OFFJ])
            y = block(int(row[T_LOFF]), mj, mj) @ x[offj:offj + mj]
            if row[T_P] >= 0:
                mp, offp = int(row[T_MP]), int(row[T_OFFP])
                y -= block(int(row[T_UOFF]), mj, mp) @ x[offp:offp + mp]
            if row[T_Q] >= 0:
                mq, offq = int(row[T_MQ]), int(row[T_OFFQ])
                y -= block(int(row[T_VOFF]), mq, mj).T @ x[offq:offq + mq]
            x[offj:offj + mj] = y
    return x


# ---- tiled solver (blocks wider than 64) -------------------------------------------------------
TILE = 64
SEG_J, SEG_P, SEG_Q = range(3)


def _strided(buf, base, rs, cs, rows, cols, what):
    """rows x cols operand with element (a, c) at buf[base + a*rs + c*cs] (bounds-checked)."""

    if rows <= 0 or cols <= 0:
        return np.zeros((max(rows, 0), max(cols, 0)))
    idx = base + np.arange(rows)[:, None] * rs + np.arange(cols)[None, :] * cs
    assert idx.min() >= 0 and idx.max() < buf.size, f"{what}: access out of range"
    return idx


class _Launch:
    """Read and write sets of the items of one launch: an item may write only what no other item
    of the launch reads or writes (the kernels rely on it; nothing orders CTAs)."""

    def __init__(self, name):
        self.name, self.items = name, []

    def item(self, reads, writes):
        cat = lambda xs: np.unique(np.concatenate([np.ravel(x) for x in xs])) if xs else np.zeros(0, int)
        self.items.append((cat(reads), cat(writes)))

    def check(self):
        owner = {}
        for n, (_, writes) in enumerate(self.items):
            for w in writes.tolist():
                assert owner.setdefault(w, n) == n, f"{self.name}: two items write one entry"
        for n, (reads, _) in enumerate(self.items):
            for r in reads.tolist():
                assert owner.get(r, n) == n, f"{self.name}: an item reads what another writes"


class _Task:
    def __init__(self, row):
        self.mj, self.offj, self.loff = int(row[T_MJ]), int(row[T_OFFJ]), int(row[T_LOFF])
        self.p = int(row[T_P])
        self.mp = int(row[T_MP]) if self.p >= 0 else 0
        self.offp, self.uoff, self.linkp = int(row[T_OFFP]), int(row[T_UOFF]), int(row[T_LINKP])
        self.q = int(row[T_Q])
        self.mq = int(row[T_MQ]) if self.q >= 0 else 0
        self.offq, self.voff, self.linkq = int(row[T_OFFQ]), int(row[T_VOFF]), int(row[T_LINKQ])
        self.fill, self.pull0, self.pull1 = int(row[T_FILL]), int(row[T_PULL0]), int(row[T_PULL1])

    def segment(self, seg, r, c):
        if seg == SEG_J:
            return self.loff + r * self.mj + c, self.mj, 1
        if seg == SEG_P:
            return self.uoff + c * self.mp + r, 1, self.mp
        return self.voff + r * self.mj + c, self.mj, 1

    def rows(self, seg):
        return (self.mj, self.mp, self.mq)[seg]


def _items(hp, r):
    b, e = hp.tranges[2 * r], hp.tranges[2 * r + 1]
    return hp.titems.reshape(-1, 4)[b:e]


SMS = 148  # multiprocessors of a B200: the tiled factorization's split rule depends on it


def panel_splits(tiles: int, systems: int, sms: int = SMS) -> int:
    """Depth splits of a panel launch, as the host code chooses them."""

    splits = 1
    while splits < 8 and tiles * systems * splits * 2 <= 2 * sms:
        splits *= 2
    return splits


def replay_factor_tiled(hp: HostPlan, values: np.ndarray, systems: int = 1, sms: int = SMS) -> np.ndarray:
    """Factor storage of one system as the tiled kernels write it (items, tiles and offsets as
    the device indexes them). Panel launches of few tiles split their depth: the partial tiles
    live in a workspace of 2 x ``sms`` tiles, indexed here past the factor storage."""

    f = np.full(hp.factor_stride, np.nan)
    widest = int(np.max(np.diff(hp.level_begin)))
    inverse_base = f.size + 2 * sms * TILE * TILE
    # factors, the split partials, then L_kk^-1 per task of a level
    space = types.SimpleNamespace(size=inverse_base + widest * TILE * TILE)
    L = hp.levels
    tasks = [_Task(r) for r in hp.tasks]
    for level in range(L):
        launch = _Launch("scatter")
        for t, r0, rows, _ in _items(hp, level):
            v = tasks[t]
            writes = [_strided(f, v.loff + r0 * v.mj, v.mj, 1, rows, v.mj, "L rows")]
            reads = []
            if v.p >= 0:
                writes.append(_strided(f, v.uoff + r0 * v.mp, v.mp, 1, rows, v.mp, "U rows"))
                if v.linkp >= 0:
                    reads.append(_strided(f, v.linkp + r0 * v.mp, v.mp, 1, rows, v.mp, "fill p"))
            if v.q >= 0:
                writes.append(_strided(f, v.voff + r0, 1, v.mj, rows, v.mq, "V cols"))
                if v.linkq >= 0:
                    reads.append(_strided(f, v.linkq + r0, 1, v.mj, rows, v.mq, "fill q"))
            launch.item(reads, writes)
        launch.check()
        for t, r0, rows, _ in _items(hp, level):  # scatter
            v = tasks[t]
            f[_strided(f, v.loff + r0 * v.mj, v.mj, 1, rows, v.mj, "L rows")] = 0.0
            if v.p >= 0:
                dst = _strided(f, v.uoff + r0 * v.mp, v.mp, 1, rows, v.mp, "U rows")
                f[dst] = 0.0 if v.linkp < 0 else f[_strided(f, v.linkp + r0 * v.mp, v.mp, 1, rows, v.mp, "fill p")]
            if v.q >= 0:
                dst = _strided(f, v.voff + r0, 1, v.mj, rows, v.mq, "V cols")
                f[dst] = 0.0 if v.linkq < 0 else f[_strided(f, v.linkq + r0, 1, v.mj, rows, v.mq, "fill q")]
            for s in range(hp.csr_ptr[v.offj + r0], hp.csr_ptr[v.offj + r0 + rows]):
                r, c = hp.csr_row[s] - v.offj, hp.csr_col[s]
                if v.offj <= c < v.offj + v.mj:
                    if c - v.offj <= r:
                        f[v.loff + r * v.mj + c - v.offj] = values[s]
                elif v.p >= 0 and v.linkp < 0 and v.offp <= c < v.offp + v.mp:
                    f[v.uoff + r * v.mp + c - v.offp] = values[s]
                elif v.q >= 0 and v.linkq < 0 and v.offq <= c < v.offq + v.mq:
                    f[v.voff + (c - v.offq) * v.mj + r] = values[s]
        panels = hp.panel_ptr[level + 1] - hp.panel_ptr[level]
        for k in range(panels):
            items = _items(hp, 3 * L + hp.panel_ptr[level] + k)
            splits = panel_splits(len(items), systems, sms)
            assert splits == 1 or len(items) * systems * splits <= 2 * sms, "split workspace overflow"
            t0 = int(hp.level_begin[level])

            def inverse(t):
                return _strided(space, inverse_base + (int(t) - t0) * TILE * TILE, TILE, 1, TILE, TILE, "inverse")

            def partial(n, z, rows, cols, splits=splits):
                # the first system's partial tile (n, z); later systems follow at items * splits tiles
                start = f.size + (n * splits + z) * TILE * TILE
                return _strided(space, start, TILE, 1, rows, cols, "partial")

            def split_panel(updates, k=k, splits=splits):
                launch = _Launch("diagonal")
                for n, ((t, _, _, _), (v, seg, i, idx, acc)) in enumerate(zip(items, updates)):
                    if seg == SEG_J and i == k:
                        ni, mk = acc.shape
                        launch.item([idx] + [partial(n, z, ni, mk) for z in range(splits)], [idx])
                launch.check()
                launch = _Launch("triangular solve")
                for n, ((t, _, _, _), (v, seg, i, idx, acc)) in enumerate(zip(items, updates)):
                    if not (seg == SEG_J and i == k):
                        mk = min(TILE, v.mj - TILE * k)
                        ni = acc.shape[0]
                        didx = _strided(f, v.loff + TILE * k * v.mj + TILE * k, v.mj, 1, mk, mk, "diag")
                        launch.item([didx, idx] + [partial(n, z, ni, mk) for z in range(splits)], [idx])
                launch.check()
                for v, seg, i, idx, acc in updates:
                    if seg == SEG_J and i == k:
                        mask = np.tril(np.ones(acc.shape, bool))
                        f[idx[mask]] -= acc[mask]
                        f[idx] = np.linalg.cholesky(np.where(mask, f[idx], f[idx].T))
                for v, seg, i, idx, acc in updates:
                    if not (seg == SEG_J and i == k):
                        mk = min(TILE, v.mj - TILE * k)
                        didx = _strided(f, v.loff + TILE * k * v.mj + TILE * k, v.mj, 1, mk, mk, "diag")
                        f[idx] = sla.solve_triangular(np.tril(f[didx]), (f[idx] - acc).T, lower=True).T

            launch = _Launch("update")
            updates = []
            for t, seg, i, _ in items:  # update launch: reads, then the item's own tile
                v = tasks[t]
                ni, mk = min(TILE, v.rows(seg) - TILE * i), min(TILE, v.mj - TILE * k)
                assert ni > 0 and mk > 0
                acc = np.zeros((ni, mk))
                reads = []
                if k > 0:
                    ia = _strided(f, *v.segment(seg, TILE * i, 0), ni, TILE * k, "A rows")
                    ib = _strided(f, *v.segment(SEG_J, TILE * k, 0), mk, TILE * k, "B rows")
                    acc += f[ia] @ f[ib].T
                    reads += [ia, ib]
                if seg == SEG_J:
                    for u in range(v.pull0, v.pull1):
                        typ, off, me = hp.pull_table[u][:3]
                        if typ == 0:
                            ia = _strided(f, off + TILE * i, 1, v.mj, ni, me, "pull U")
                            ib = _strided(f, off + TILE * k, 1, v.mj, mk, me, "pull U")
                        else:
                            ia = _strided(f, off + TILE * i * me, me, 1, ni, me, "pull V")
                            ib = _strided(f, off + TILE * k * me, me, 1, mk, me, "pull V")
                        acc += f[ia] @ f[ib].T
                        reads += [ia, ib]
                idx = _strided(f, *v.segment(seg, TILE * i, TILE * k), ni, mk, "C tile")
                updates.append((v, seg, i, idx, acc))
                if splits == 1:
                    launch.item(reads, [idx, inverse(t)] if seg == SEG_J and i == k else [idx])
                    continue
                for z in range(splits):
                    launch.item(reads, [partial(len(updates) - 1, z, ni, mk)])
            launch.check()
            if splits > 1:
                split_panel(updates)
                continue
            for v, seg, i, idx, acc in updates:
                if seg == SEG_J and i == k:  # lower part, then the in-place Cholesky of the tile
                    mask = np.tril(np.ones(acc.shape, bool))
                    f[idx[mask]] -= acc[mask]
                    f[idx] = np.linalg.cholesky(np.where(mask, f[idx], f[idx].T))
                else:
                    f[idx] -= acc
            launch = _Launch("triangular solve")
            solves = []
            for t, seg, i, _ in items:
                v = tasks[t]
                if seg == SEG_J and i == k:
                    continue
                mk = min(TILE, v.mj - TILE * k)
                didx = _strided(f, v.loff + TILE * k * v.mj + TILE * k, v.mj, 1, mk, mk, "diag")
                ni = min(TILE, v.rows(seg) - TILE * i)
                idx = _strided(f, *v.segment(seg, TILE * i, TILE * k), ni, mk, "tile")
                launch.item([inverse(t)], [idx])
                solves.append((didx, idx))
            launch.check()
            for didx, idx in solves:
                f[idx] = sla.solve_triangular(np.tril(f[didx]), f[idx].T, lower=True).T
        launch = _Launch("fill")
        fills = []
        for t, qi, pi, _ in _items(hp, L + level):
            v = tasks[t]
            nq, npp = min(TILE, v.mq - TILE * qi), min(TILE, v.mp - TILE * pi)
            ia = _strided(f, v.voff + TILE * qi * v.mj, v.mj, 1, nq, v.mj, "fill V")
            ib = _strided(f, v.uoff + TILE * pi, 1, v.mp, npp, v.mj, "fill U")
            io = _strided(f, v.fill + TILE * qi * v.mp + TILE * pi, v.mp, 1, nq, npp, "fill")
            launch.item([ia, ib], [io])
            fills.append((ia, ib, io))
        launch.check()
        for ia, ib, io in fills:
            f[io] = -(f[ia] @ f[ib].T)
    return f


def replay_solve_tiled(hp: HostPlan, f: np.ndarray, rhs: np.ndarray) -> np.ndarray:
    """Forward and backward substitution of the tiled kernels on rhs [N][ncols] (solver order)."""

    x = np.array(rhs, dtype=float)
    L = hp.levels
    tasks = [_Task(r) for r in hp.tasks]

    def lj(v):
        return f[_strided(f, v.loff, v.mj, 1, v.mj, v.mj, "L_j")]

    for level in range(L):
        for t, i, _, _ in _items(hp, 2 * L + level):
            v = tasks[t]
            ni = min(TILE, v.mj - TILE * i)
            rows = slice(v.offj + TILE * i, v.offj + TILE * i + ni)
            for u in range(v.pull0, v.pull1):
                typ, off, me, eoff = hp.pull_table[u][:4]
                if typ == 0:
                    a = f[_strided(f, off + TILE * i, 1, v.mj, ni, me, "pull U")]
                else:
                    a = f[_strided(f, off + TILE * i * me, me, 1, ni, me, "pull V")]
                x[rows] -= a @ x[eoff:eoff + me]
        for t in range(hp.level_begin[level], hp.level_begin[level + 1]):
            v = tasks[t]
            block = slice(v.offj, v.offj + v.mj)
            x[block] = sla.solve_triangular(lj(v), x[block], lower=True)
            if level == L - 1:
                x[block] = sla.solve_triangular(lj(v).T, x[block], lower=False)
    for level in range(L - 2, -1, -1):
        for t, i, _, _ in _items(hp, 2 * L + level):
            v = tasks[t]
            ni = min(TILE, v.mj - TILE * i)
            rows = slice(v.offj + TILE * i, v.offj + TILE * i + ni)
            if v.p >= 0:
                a = f[_strided(f, v.uoff + TILE * i * v.mp, v.mp, 1, ni, v.mp, "U_p")]
                x[rows] -= a @ x[v.offp:v.offp + v.mp]
            if v.q >= 0:
                a = f[_strided(f, v.voff + TILE * i, 1, v.mj, ni, v.mq, "V_q")]
                x[rows] -= a @ x[v.offq:v.offq + v.mq]
        for t in range(hp.level_begin[level], hp.level_begin[level + 1]):
            v = tasks[t]
            block = slice(v.offj, v.offj + v.mj)
            x[block] = sla.solve_triangular(lj(v).T, x[block], lower=False)
    return x
