"""Many CSR matrices of uneven size: SpMV and SpMM for all of them in one graph launch.

The matrices become one block-diagonal CSR (prepare, once): row, column and
nonzero offsets per matrix, indices shifted by the column offset.  One SpMV
and one SpMM over the combined matrix then compute every y_i = A_i x_i and
C_i = A_i B_i, because the unit plan cuts work across matrix boundaries like
any other row boundary: large and small matrices share the same warps.

A step is either the SpMV and the SpMM launches, or -- for real values with a
narrow B (N * sizeof(value) <= 256 bytes) -- ONE kernel: the narrow-row SpMM
kernel whose lanes also sum y = A x from x[col] gathered beside B's row
(``fsb_spmm_spmv_csr``), which reads the matrix once for both products.  The
autotuner times both and keeps the faster; untuned, the step is unfused.

Inputs and outputs live in static device buffers (``x``, ``B``, ``y``, ``C``)
with one view per matrix; ``capture()`` records the step in a CUDA graph and
``run()`` replays it, so a step is a single host launch.

``tune()`` is the schedule autotuner: it times candidate plan parameters (the
row-block window ``cap`` and the long-row chunk of the SpMV and the SpMM
plans, and for the best SpMM shape the persistent grid against one work item
per warp) and the fused step on this batch and keeps the fastest schedule;
results are cached per batch signature (dtype, width, row-length histogram)
in memory and, when a path is given, in a JSON file.
"""

import json
import math
import os

import torch

from .. import _native as nat
from . import _csr

# SpMV windows are given as fractions of the value type's largest window
# (fsb_spmv_default_cap: 224 for 2- and 4-byte real types, 128 otherwise).
SPMV_CANDIDATES = ({"cap": 1, "chunk": 512}, {"cap": 2, "chunk": 512}, {"cap": 4, "chunk": 512},
                   {"cap": 1, "chunk": 1024})
SPMM_CANDIDATES = ({"cap": 64, "chunk": 256}, {"cap": 32, "chunk": 256}, {"cap": 16, "chunk": 256},
                   {"cap": 64, "chunk": 512})
_TUNE_CACHE = {}


def _signature(dtype, n_dense, row_lengths):
    """Batch signature: dtype, dense width and a log2 histogram of row lengths."""
    hist = torch.bincount(torch.log2(row_lengths.double().clamp_min(1)).floor().long(), minlength=20)[:20]
    total = max(int(row_lengths.numel()), 1)
    shape = tuple(round(float(v) / total, 3) for v in hist.tolist())
    return f"{dtype}|N{n_dense}|rows~2^{round(math.log2(total))}|{shape}"


class BatchedCsr:
    """Block-diagonal concatenation of CSR matrices with static x / B / y / C buffers."""

    def __init__(self, matrices, n_dense=16, dtype=None, device=None):
        """``matrices``: list of ``(data, indices, indptr, shape)`` CUDA tensors."""
        if not matrices:
            raise ValueError("matrices must be a non-empty list")
        device = device or matrices[0][0].device
        dtype = dtype or matrices[0][0].dtype
        if dtype not in nat.DTYPE_CODE:
            raise TypeError(f"unsupported value dtype {dtype}")
        datas, inds, ptrs = [], [], []
        self.row_off, self.col_off, self.nnz_off = [0], [0], [0]
        for data, indices, indptr, shape in matrices:
            m, k = int(shape[0]), int(shape[1])
            if indptr.numel() != m + 1 or data.numel() != indices.numel():
                raise ValueError("each matrix needs indptr of length n_rows+1 and data / indices of length nnz")
            facts = _csr.inspect_csr(indices, indptr, m, indices.numel())
            if facts["first"] != 0 or facts["last"] != indices.numel() or facts["decreasing"]:
                raise ValueError("indptr must start at 0, end at nnz and be nondecreasing")
            if indices.numel() and (facts["min_col"] < 0 or facts["max_col"] >= k):
                raise IndexError("indices out of range for n_cols")
            datas.append(data.to(device=device, dtype=dtype))
            inds.append(indices.to(device=device, dtype=torch.int32) + self.col_off[-1])
            ptrs.append(indptr[:-1].to(device=device, dtype=torch.int64) + self.nnz_off[-1])
            self.row_off.append(self.row_off[-1] + m)
            self.col_off.append(self.col_off[-1] + k)
            self.nnz_off.append(self.nnz_off[-1] + int(indices.numel()))
        self.count = len(matrices)
        self.n_rows, self.n_cols, self.nnz = self.row_off[-1], self.col_off[-1], self.nnz_off[-1]
        if self.n_rows >= 2**31 - 1 or self.n_cols >= 2**31 - 1:
            raise ValueError("the combined matrix must have fewer than 2^31 rows and columns")
        self.data = torch.cat(datas)
        self.indices = torch.cat(inds)
        self.indptr = torch.cat(ptrs + [torch.tensor([self.nnz], dtype=torch.int64, device=device)])
        self.dtype, self.device, self.n_dense = dtype, device, int(n_dense)
        self.x = torch.zeros(self.n_cols, dtype=dtype, device=device)
        self.B = torch.zeros(self.n_cols, self.n_dense, dtype=dtype, device=device)
        self.y = torch.empty(self.n_rows, dtype=dtype, device=device)
        self.C = torch.empty(self.n_rows, self.n_dense, dtype=dtype, device=device)
        self.spmv_cfg = {"cap": int(nat.lib().fsb_spmv_default_cap(nat.dtype_code(dtype))), "chunk": 512}
        self.spmm_cfg = dict(SPMM_CANDIDATES[0])
        self._spmv_plan = self._spmm_plan = None
        self._graph = None
        self.tuning = None
        self.fused = False  # the one-kernel step, when the autotuner picks it

    # ------------------------------------------------------------ views
    def x_view(self, i):
        return self.x[self.col_off[i]:self.col_off[i + 1]]

    def B_view(self, i):
        return self.B[self.col_off[i]:self.col_off[i + 1]]

    def y_view(self, i):
        return self.y[self.row_off[i]:self.row_off[i + 1]]

    def C_view(self, i):
        return self.C[self.row_off[i]:self.row_off[i + 1]]

    # ------------------------------------------------------------ launches
    def _spmv_plan_get(self):
        if self._spmv_plan is None:
            self._spmv_plan = _csr.NativeSpmvPlan(self.indptr, self.n_rows, self.dtype, cap=self.spmv_cfg["cap"],
                                                  chunk_nnz=self.spmv_cfg["chunk"])
        return self._spmv_plan

    def _spmm_plan_get(self):
        if self._spmm_plan is None:
            self._spmm_plan = _csr.SpmmPlan(self.indptr, self.n_rows, self.dtype, cap=self.spmm_cfg["cap"],
                                            chunk_nnz=self.spmm_cfg["chunk"])
        return self._spmm_plan

    def _plans(self):
        return self._spmv_plan_get(), self._spmm_plan_get()

    def _launch_spmv(self, plan):
        nat.check(
            nat.lib().fsb_spmv_csr(nat.dtype_code(self.dtype), nat.ptr(self.data), nat.ptr(self.indices), 0,
                                   nat.ptr(self.indptr), 1, self.n_rows, self.n_cols, nat.ptr(self.x), nat.ptr(self.y),
                                   plan.struct_ref(), nat.stream_of(self.device)),
            "fsb_spmv_csr",
        )

    def _launch_spmm(self, plan, persistent=None):
        if persistent is None:
            persistent = bool(self.spmm_cfg.get("persistent", False))
        _csr.spmm(self.data, self.indices, self.indptr, self.n_rows, self.n_cols, self.B, plan, self.C,
                  persistent=persistent)

    def _launch_fused(self, plan, persistent=None):
        if persistent is None:
            persistent = bool(self.spmm_cfg.get("persistent", False))
        return _csr.spmm_spmv(self.data, self.indices, self.indptr, self.n_rows, self.n_cols, self.B, plan, self.C,
                              self.x, self.y, persistent=persistent)

    def step(self):
        """y = A x and C = A B over the whole batch (no graph): the fused launch when
        selected and applicable, else the SpMV and the SpMM launches."""
        if self.fused:
            if self._launch_fused(self._spmm_plan_get()):
                return
            self.fused = False
        self._launch_spmv(self._spmv_plan_get())
        self._launch_spmm(self._spmm_plan_get())

    # ------------------------------------------------------------ autotuner
    def _time(self, fn, reps=5):
        for _ in range(2):
            fn()
        torch.cuda.synchronize(self.device)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(reps):
            fn()
        end.record()
        end.synchronize()
        return start.elapsed_time(end) / reps

    def tune(self, cache_path=None):
        """Pick the fastest SpMV and SpMM plan parameters for this batch; returns the report."""
        sig = _signature(self.dtype, self.n_dense, self.indptr[1:] - self.indptr[:-1])
        cached = _TUNE_CACHE.get(sig)
        if cached is None and cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                cached = json.load(f).get(sig)
        if cached is not None:
            self.spmv_cfg, self.spmm_cfg = dict(cached["spmv"]), dict(cached["spmm"])
            self.fused = bool(cached.get("fused", False))
            self._spmv_plan = self._spmm_plan = None
            self._graph = None
            self.tuning = dict(cached, source="cache")
            return self.tuning
        report = {"signature": sig, "spmv_trials": [], "spmm_trials": [], "fused_trials": []}
        best_v = best_m = best_f = None
        max_cap = int(nat.lib().fsb_spmv_default_cap(nat.dtype_code(self.dtype)))
        for frac in SPMV_CANDIDATES:
            cfg = {"cap": max_cap // frac["cap"], "chunk": frac["chunk"]}
            plan = _csr.NativeSpmvPlan(self.indptr, self.n_rows, self.dtype, cap=cfg["cap"], chunk_nnz=cfg["chunk"])
            ms = self._time(lambda: self._launch_spmv(plan))
            report["spmv_trials"].append(dict(cfg, ms=round(ms, 5)))
            if best_v is None or ms < best_v[1]:
                best_v = (cfg, ms)
        fusable = self._launch_fused(self._spmm_plan_get(), persistent=False)
        # each plan shape with one work item per warp, then the best one also on the
        # persistent grid (same results, another schedule of the same items)
        for cfg in SPMM_CANDIDATES:
            cfg = dict(cfg, persistent=False)
            plan = _csr.SpmmPlan(self.indptr, self.n_rows, self.dtype, cap=cfg["cap"], chunk_nnz=cfg["chunk"])
            ms = self._time(lambda: self._launch_spmm(plan, False))
            report["spmm_trials"].append(dict(cfg, ms=round(ms, 5)))
            if best_m is None or ms < best_m[1]:
                best_m = (cfg, ms)
            if fusable:
                ms = self._time(lambda: self._launch_fused(plan, False))
                report["fused_trials"].append(dict(cfg, ms=round(ms, 5)))
                if best_f is None or ms < best_f[1]:
                    best_f = (cfg, ms)
        def persistent_trial(best, launch, trials):
            if best is None:
                return best
            cfg = dict(best[0], persistent=True)
            plan = _csr.SpmmPlan(self.indptr, self.n_rows, self.dtype, cap=cfg["cap"], chunk_nnz=cfg["chunk"])
            ms = self._time(lambda: launch(plan, True))
            report[trials].append(dict(cfg, ms=round(ms, 5)))
            return (cfg, ms) if ms < best[1] else best

        best_m = persistent_trial(best_m, self._launch_spmm, "spmm_trials")
        best_f = persistent_trial(best_f, self._launch_fused, "fused_trials")
        self.fused = best_f is not None and best_f[1] < best_v[1] + best_m[1]
        self.spmv_cfg = dict(best_v[0])
        self.spmm_cfg = dict(best_f[0] if self.fused else best_m[0])
        fused = self.fused
        self._spmv_plan = self._spmm_plan = None
        self._graph = None
        report.update(spmv=self.spmv_cfg, spmm=self.spmm_cfg, fused=bool(fused))
        _TUNE_CACHE[sig] = report
        if cache_path:
            data = {}
            if os.path.exists(cache_path):
                with open(cache_path) as f:
                    data = json.load(f)
            data[sig] = report
            with open(cache_path, "w") as f:
                json.dump(data, f, indent=1)
        self.tuning = dict(report, source="measured")
        return self.tuning

    # ------------------------------------------------------------ graph
    def capture(self):
        """Record the batch step in a CUDA graph on a side stream."""
        self.step()  # decides fused / unfused; scratch for this width exists before capture
        torch.cuda.synchronize(self.device)
        stream = torch.cuda.Stream(device=self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(stream):
            with torch.cuda.graph(graph, stream=stream):
                self.step()
        torch.cuda.synchronize(self.device)
        self._graph = graph
        return graph

    def run(self):
        """Replay the captured step on the current stream (captures first if needed)."""
        if self._graph is None:
            self.capture()
        self._graph.replay()
        return self.y, self.C

    def bytes_models(self):
        """(SpMV bytes, SpMM compulsory bytes, SpMM gather bytes) per step for this batch."""
        s = self.data.element_size()
        n = self.n_dense
        spmv = self.nnz * (s + 4) + (self.n_rows + self.count) * 8 + self.n_cols * s + self.n_rows * s
        spmm_c = self.nnz * (s + 4) + self.n_cols * n * s + self.n_rows * n * s
        spmm_g = self.nnz * (s + 4) + self.nnz * n * s + self.n_rows * n * s
        return spmv, spmm_c, spmm_g
