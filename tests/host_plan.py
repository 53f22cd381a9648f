"""CPU access to the plan builder of adtlert_b200 and a NumPy replay of its device schedule.

``compile_shim`` builds ``tests/native/host_plan_shim.cpp`` together with the library's own
``plan_host.cpp`` (no CUDA); ``HostPlan`` exposes the tables; the ``replay_*`` functions execute
the solver and assembly tables exactly as the CUDA kernels index them (same offsets, same block
shapes), asserting that every access stays inside its buffer.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np
import scipy.linalg as sla

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "ad-tlert_b200" / "csrc"
BUILD = ROOT / "tests" / "_build"

T_J, T_MJ, T_OFFJ, T_LOFF, T_P, T_MP, T_OFFP, T_UOFF, T_LINKP, T_Q, T_MQ, T_OFFQ, T_VOFF, T_LINKQ, T_FILL, T_PULL0, T_PULL1 = range(17)
T_FIELDS = 17
P_TYPE, P_OFF, P_ME, P_EOFF = range(4)

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
            for name in ("N", "nnz", "nb", "max_m", "levels", "RS", "R", "rdofs", "factor_stride", "contributions"):
                setattr(self, name, int(lib.shim_scalar(handle, name.encode())))
            for name in ("perm", "iperm", "level_begin", "csr_ptr", "csr_col", "csr_row", "contrib_ptr", "contrib",
                         "task_rows", "pulls", "features", "fscale", "pair_ptr", "pair_list", "rcv_dofs", "rcv_w",
                         "rdof_ptr", "rdof_rcv", "rdof_dof", "rdof_w", "cdofs", "bd", "cell_bptr", "cell_blist",
                         "model_ptr", "model_list", "k2", "bowners", "fixed"):
                size = lib.shim_table(handle, name.encode(), None)
                out = np.empty(size, dtype=_TYPES.get(name, np.int32))
                lib.shim_table(handle, name.encode(), out.ctypes.data_as(ctypes.c_void_p))
                setattr(self, name, out)
            self.tasks = self.task_rows.reshape(-1, T_FIELDS)
            self.pull_table = self.pulls.reshape(-1, 4)

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


def replay_factor(hp: HostPlan, values: np.ndarray) -> np.ndarray:
    """Factor storage of one system, written as factor_level_kernel writes it."""

    stride = hp.factor_stride
    f = np.full(stride, np.nan)
    written = np.zeros(stride, dtype=bool)

    def store(offset, block, what):
        _check(offset, block.size, stride, what)
        assert not written[offset:offset + block.size].any(), f"{what}: storage written twice"
        f[offset:offset + block.size] = block.reshape(-1)
        written[offset:offset + block.size] = True

    def load(offset, rows, cols, what):
        _check(offset, rows * cols, stride, what)
        block = f[offset:offset + rows * cols].reshape(rows, cols)
        assert np.all(np.isfinite(block)), f"{what}: read before written"
        return block

    for level in range(hp.levels):
        for t in range(hp.level_begin[level], hp.level_begin[level + 1]):
            row = hp.tasks[t]
            mj, offj = int(row[T_MJ]), int(row[T_OFFJ])
            p, mp, offp = int(row[T_P]), int(row[T_MP]), int(row[T_OFFP])
            q, mq, offq = int(row[T_Q]), int(row[T_MQ]), int(row[T_OFFQ])
            assert 0 < mj <= 64 and (p < 0 or 0 < mp <= 64) and (q < 0 or 0 < mq <= 64)
            p_csr, q_csr = p >= 0 and row[T_LINKP] < 0, q >= 0 and row[T_LINKQ] < 0
            dm, ap, aq = np.zeros((mj, mj)), np.zeros((mj, max(mp, 0))), np.zeros((max(mq, 0), mj))
            for s in range(hp.csr_ptr[offj], hp.csr_ptr[offj + mj]):
                r, c = hp.csr_row[s] - offj, hp.csr_col[s]
                assert 0 <= r < mj
                if offj <= c < offj + mj:
                    dm[r, c - offj] = values[s]
                elif p_csr and offp <= c < offp + mp:
                    ap[r, c - offp] = values[s]
                elif q_csr and offq <= c < offq + mq:
                    aq[c - offq, r] = values[s]
            if p >= 0 and not p_csr:
                ap = load(int(row[T_LINKP]), mj, mp, "link p").copy()
            if q >= 0 and not q_csr:
                aq = load(int(row[T_LINKQ]), mq, mj, "link q").copy()
            for u in range(row[T_PULL0], row[T_PULL1]):
                kind, off, me = (int(v) for v in hp.pull_table[u, :3])
                if kind == 0:
                    U = load(off, me, mj, "pull U")
                    dm -= U.T @ U
                else:
                    V = load(off, mj, me, "pull V")
                    dm -= V @ V.T
            L = np.linalg.cholesky(np.tril(dm) + np.tril(dm, -1).T)
            store(int(row[T_LOFF]), L, "L")
            if p >= 0:
                U = sla.solve_triangular(L, ap, lower=True)
                store(int(row[T_UOFF]), U, "U")
            if q >= 0:
                V = sla.solve_triangular(L, aq.T, lower=True).T
                store(int(row[T_VOFF]), V, "V")
            if p >= 0 and q >= 0:
                store(int(row[T_FILL]), -V @ U, "fill")
    return f


def replay_solve(hp: HostPlan, f: np.ndarray, rhs: np.ndarray) -> np.ndarray:
    """Solution of one system for rhs (N, nrhs) in solver order, as the level kernels compute it."""

    x = rhs.astype(float).copy()

    def block(off, rows, cols):
        return f[off:off + rows * cols].reshape(rows, cols)

    for level in range(hp.levels):
        root = level == hp.levels - 1
        for t in range(hp.level_begin[level], hp.level_begin[level + 1]):
            row = hp.tasks[t]
            mj, offj = int(row[T_MJ]), int(row[T_OFFJ])
            b = x[offj:offj + mj].copy()
            for u in range(row[T_PULL0], row[T_PULL1]):
                kind, off, me, eoff = (int(v) for v in hp.pull_table[u])
                y = x[eoff:eoff + me]
                b -= (block(off, me, mj).T @ y) if kind == 0 else (block(off, mj, me) @ y)
            L = block(int(row[T_LOFF]), mj, mj)
            b = sla.solve_triangular(L, b, lower=True)
            if root:
                b = sla.solve_triangular(L.T, b, lower=False)
            x[offj:offj + mj] = b
    for level in range(hp.levels - 2, -1, -1):
        for t in range(hp.level_begin[level], hp.level_begin[level + 1]):
            row = hp.tasks[t]
            mj, offj = int(row[T_MJ]), int(row[T_OFFJ])
            y = x[offj:offj + mj].copy()
            if row[T_P] >= 0:
                mp, offp = int(row[T_MP]), int(row[T_OFFP])
                y -= block(int(row[T_UOFF]), mj, mp) @ x[offp:offp + mp]
            if row[T_Q] >= 0:
                mq, offq = int(row[T_MQ]), int(row[T_OFFQ])
                y -= block(int(row[T_VOFF]), mq, mj).T @ x[offq:offq + mq]
            x[offj:offj + mj] = sla.solve_triangular(block(int(row[T_LOFF]), mj, mj).T, y, lower=False)
    return x
