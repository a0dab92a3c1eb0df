"""Benchmark of the CSR hot path on B200.

Default workload: plain CSR SpMV y = A x, float32 values, int32 column
indices, on the 2,000,000 x 2,000,000 Zipf(2) matrix (row length
min(50000, ceil(2.887 Z)), ~39M nonzeros, seed 1) -- the configuration the
headline metric "CSR SpMV/SpMM GB/s vs HBM peak" is quoted on.  A step is one
SpMV over the whole matrix.

  value     algorithmic GB/s with A, x resident in HBM (CUDA events, L2
            flushed between steps), summed over ranks / max rank time
  e2e       the same metric through the public API with x copied from pinned
            host memory and y read back every step (copies of neighbouring
            steps overlap the SpMV)
  roofline  algorithmic bytes per launch / mean launch time vs measured HBM peak
  cpu_baseline  the CPU oracle on the host cores, bounded sample

``--impl reference`` times the reference's CPU path for this operator:
torch.sparse.mm on a CPU sparse_csr_tensor, fp32 values summed in fp64 as the
reference's own fp32 tests compute their reference, with all host threads.
The C restatement of the same semantics (oracle/) is reported beside it.
Multi-GPU (torchrun): the headline SpMV splits the matrix by rows across the
ranks (ShardedCsr, strong scaling, no data-path collective); the other
``--case`` workloads run one independent replica per rank (weak scaling).
"""

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "CSR SpMV/SpMM GB/s vs HBM peak; bf16+autograd vs fp32 plain at stated error"


# ---------------------------------------------------------------- helpers

def _measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _measured_bf16_tflops():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f).get("bf16_tflops", 1590.0))
    return 1590.0


def _ncu_traffic(workload):
    path = os.path.join(REPO, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get(workload)


class ClockSampler:
    """Polls SM clocks and clock-event reasons through NVML (read-only) every ~1 ms.

    Samples carry host timestamps; ``mark`` records the bounds of the timed
    region, and ``stop`` summarises the samples taken inside it (widened to
    the whole measured phase when the timed region is too short to hold a
    few samples).  Reports None when NVML is unusable.
    """

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, cuda_index):
        self.cuda_index = int(cuda_index)
        self.samples = []  # (t, sm_mhz, max_mhz, reasons bitmask)
        self.marks = {}
        self._stop = threading.Event()
        self.thread = None
        self.source = None

    def start(self):
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            idx = torch.cuda._get_nvml_device_index(self.cuda_index)
            self._nvml = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self._max = float(pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM))
            self._bits = {name: getattr(pynvml, attr, 0) for name, attr in self.REASONS}
            self.source = "nvml"
        except Exception:
            self.source = None
            return
        self.thread = threading.Thread(target=self._poll, daemon=True)
        self.thread.start()
        t0 = time.monotonic()
        while not self.samples and time.monotonic() - t0 < 2.0:
            time.sleep(0.001)

    def _poll(self):
        nv, h = self._nvml, self._h
        while not self._stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
            except Exception:
                break
            self.samples.append((time.monotonic(), sm, self._max, rs))
            time.sleep(0.001)

    def mark(self, name):
        self.marks[name] = time.monotonic()

    def stop(self):
        if self.thread is None:
            return None
        self._stop.set()
        self.thread.join(timeout=2)
        try:
            self._nvml.nvmlShutdown()
        except Exception:
            pass
        t0, t1 = self.marks.get("timed_start", 0.0), self.marks.get("timed_end", float("inf"))
        window = "timed"
        sel = [s for s in self.samples if t0 <= s[0] <= t1]
        if len(sel) < 3:
            t1 = self.marks.get("phase_end", t1)
            sel = [s for s in self.samples if t0 <= s[0] <= t1]
            window = "timed+e2e (timed region shorter than the poll interval)"
        if not sel:
            return None
        reasons = sorted(name for name, bit in self._bits.items() if bit and any(s[3] & bit for s in sel))
        return {"sm_mhz": statistics.median(s[1] for s in sel), "sm_max_mhz": max(s[2] for s in sel),
                "reasons": reasons, "samples": len(sel), "window": window, "source": self.source}


# ---------------------------------------------------------------- the reference's CPU path

class TorchCpuSpmv:
    """y = A x on the host cores through torch.sparse.mm on a CPU sparse_csr_tensor: the
    reference's CPU path.  fp32 values and x are summed in fp64 and y is rounded back to
    fp32, as the reference's fp32 tests form their reference (tests/pytest/
    test_spmm_csr_accuracy.py:108-117, test_spmv_csr_accuracy.py:52-59).  The fp64 copy
    of A is made once (the reference caches its fp64 copy of the values too,
    sparse_operations/spmv_csr.py:138-144); x is widened every step."""

    def __init__(self, c, nthreads=None):
        import torch

        self.torch = torch
        self.nthreads = int(nthreads or os.cpu_count() or 1)
        torch.set_num_threads(self.nthreads)
        self.A64 = torch.sparse_csr_tensor(torch.from_numpy(c["indptr"]), torch.from_numpy(c["indices"]),
                                           torch.from_numpy(c["data"].astype(np.float64)), size=c["shape"])
        self.x = torch.from_numpy(c["x"])

    def step(self):
        torch = self.torch
        return torch.sparse.mm(self.A64, self.x.double()[:, None])[:, 0].float()


def _wall_per_step(fn, budget_s, max_reps=400):
    """Repeat fn() until ~budget_s seconds have passed; return (seconds per step, reps)."""
    fn()
    reps, t0 = 0, time.perf_counter()
    while True:
        fn()
        reps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or reps >= max_reps:
            return el / reps, reps


def spmv_zipf_config(M, K, nnz):
    return {"workload": "spmv_csr_zipf2_2Mx2M_f32", "rows": M, "cols": K, "nnz": nnz,
            "row_length": "min(50000, ceil(2.887*Z)), Z~Zipf(2) truncated at 50000",
            "index_dtype": "int32", "indptr_dtype": "int64", "seed": 1,
            "l2": "flushed between timed steps (256 MiB write, then a 50 us device spin that covers the host call)"}


# ---------------------------------------------------------------- workloads

class SpmvZipf:
    name = "spmv_csr_zipf2_2Mx2M_f32"
    dtype = "f32"

    def __init__(self, device, seed=1):
        import torch

        import flagsparse_b200 as fs
        from flagsparse_b200 import workloads

        self.torch = torch
        self.fs = fs
        c = workloads.zipf_csr(n=2_000_000, seed=seed, dtype=np.float32)
        self.host = c
        self.M, self.K = c["shape"]
        self.nnz = int(c["indices"].size)
        self.device = device
        self.data = torch.from_numpy(c["data"]).to(device)
        self.indices = torch.from_numpy(c["indices"]).to(device)
        self.indptr = torch.from_numpy(c["indptr"]).to(device)
        self.x = torch.from_numpy(c["x"]).to(device)
        self.prepared = fs.prepare_spmv_csr(self.data, self.indices, self.indptr, c["shape"])
        self.y = torch.empty(self.M, dtype=torch.float32, device=device)
        # pinned host buffers for the end-to-end leg
        self.x_host = torch.from_numpy(c["x"]).pin_memory()
        self.y_host = torch.empty(self.M, dtype=torch.float32).pin_memory()
        self.x_dev2 = torch.empty_like(self.x)
        # double-buffered device and host copies for the pipelined end-to-end leg
        self.x_buf = [torch.empty_like(self.x) for _ in range(2)]
        self.y_buf = [torch.empty_like(self.y) for _ in range(2)]
        self.y_hosts = [torch.empty(self.M, dtype=torch.float32).pin_memory() for _ in range(2)]
        self.s_in = torch.cuda.Stream(device=device)
        self.s_out = torch.cuda.Stream(device=device)

    def config(self):
        return dict(spmv_zipf_config(self.M, self.K, self.nnz), workload=self.name)

    def alg_bytes(self):
        # values + column indices + row pointers + x once + y once
        return self.nnz * (4 + 4) + (self.M + 1) * 8 + self.K * 4 + self.M * 4

    def step(self):
        self.fs.flagsparse_spmv_csr(x=self.x, prepared=self.prepared, out=self.y)

    def e2e_step(self):
        self.x_dev2.copy_(self.x_host, non_blocking=True)
        self.fs.flagsparse_spmv_csr(x=self.x_dev2, prepared=self.prepared, out=self.y)
        self.y_host.copy_(self.y, non_blocking=True)

    def e2e_run(self, steps):
        """``steps`` end-to-end SpMVs, pipelined over three streams.

        Step i uploads x into buffer i%2 on the upload stream, runs the SpMV on
        the current stream and downloads y from buffer i%2 on the download
        stream, so the upload of step i+1 and the download of step i-1 overlap
        the SpMV of step i.  Every step still moves its full x in and y out."""
        torch = self.torch
        cur = torch.cuda.current_stream()
        self.s_in.wait_stream(cur)
        self.s_out.wait_stream(cur)
        done_spmv, done_out = [None, None], [None, None]
        for i in range(steps):
            b = i & 1
            with torch.cuda.stream(self.s_in):
                if done_spmv[b] is not None:
                    self.s_in.wait_event(done_spmv[b])  # buffer b's previous SpMV has read x
                self.x_buf[b].copy_(self.x_host, non_blocking=True)
                ev_in = torch.cuda.Event()
                ev_in.record(self.s_in)
            cur.wait_event(ev_in)
            if done_out[b] is not None:
                cur.wait_event(done_out[b])  # buffer b's previous y is on the host
            self.fs.flagsparse_spmv_csr(x=self.x_buf[b], prepared=self.prepared, out=self.y_buf[b])
            ev_spmv = torch.cuda.Event()
            ev_spmv.record(cur)
            done_spmv[b] = ev_spmv
            with torch.cuda.stream(self.s_out):
                self.s_out.wait_event(ev_spmv)
                self.y_hosts[b].copy_(self.y_buf[b], non_blocking=True)
                ev_out = torch.cuda.Event()
                ev_out.record(self.s_out)
                done_out[b] = ev_out
        cur.wait_stream(self.s_out)

    def e2e_bytes(self):
        return self.K * 4, self.M * 4

    def launches_per_step(self):
        # row-block units and long-row chunks run as separate launches
        p = self.prepared.native_plan()
        return int(p.n_block_units > 0) + int(p.n_units > p.n_block_units)

    def cpu_run(self, nthreads):
        from oracle import oracle

        c = self.host
        return oracle.spmv_f32_acc64(c["indptr"], c["indices"], c["data"], c["x"], nthreads=nthreads)


class SpmvZipfSharded(SpmvZipf):
    """The headline SpMV split across ranks by rows (flagsparse_b200.distributed.ShardedCsr):
    each rank multiplies its block of rows (about nnz / world nonzeros) by the whole x and
    keeps its rows of y.  The total work is fixed (strong scaling); value = the whole
    matrix's bytes / the slowest rank's time."""

    pipelined = False  # end-to-end steps run serially (upload, SpMV, download)

    def __init__(self, device, rank, world, seed=1):
        import torch

        import flagsparse_b200 as fs
        from flagsparse_b200 import distributed as fsd
        from flagsparse_b200 import workloads

        self.torch, self.fs = torch, fs
        c = workloads.zipf_csr(n=2_000_000, seed=seed, dtype=np.float32)
        self.host = c
        self.M, self.K = c["shape"]
        self.nnz = int(c["indices"].size)
        self.device = device
        self.sh = fsd.ShardedCsr(torch.from_numpy(c["data"]), torch.from_numpy(c["indices"]),
                                 torch.from_numpy(c["indptr"]), c["shape"], rank=rank, world_size=world,
                                 device=device)
        self.prepared = self.sh.prepared
        self.rows = self.sh.row_end - self.sh.row_begin
        self.local_nnz = int(self.sh.indices.numel())
        self.x = torch.from_numpy(c["x"]).to(device)
        self.y = torch.empty(self.rows, dtype=torch.float32, device=device)
        self.x_host = torch.from_numpy(c["x"]).pin_memory()
        self.x_dev2 = torch.empty_like(self.x)
        self.y_host = torch.empty(self.rows, dtype=torch.float32).pin_memory()

    def config(self):
        return dict(super().config(), split="rows balanced by nonzeros, x replicated, y row-sharded")

    def alg_bytes(self):
        # this rank's share: its values, columns, row pointers, the whole x and its rows of y
        return self.local_nnz * 8 + (self.rows + 1) * 8 + self.K * 4 + self.rows * 4

    def total_bytes(self):
        return self.nnz * (4 + 4) + (self.M + 1) * 8 + self.K * 4 + self.M * 4

    def step(self):
        self.sh.spmv(self.x, out=self.y)

    def e2e_step(self):
        self.x_dev2.copy_(self.x_host, non_blocking=True)
        self.sh.spmv(self.x_dev2, out=self.y)
        self.y_host.copy_(self.y, non_blocking=True)

    def e2e_bytes(self):
        return self.K * 4, self.rows * 4


class SpmvGatherFloor(SpmvZipf):
    """The x-gather floor of the headline SpMV (fsb_spmv_gather_floor): the fp64 sum of
    data[i] * x[indices[i]] over all 38.9 M nonzeros of the 2M Zipf(2) matrix, with the
    SpMV's own load kinds but no row structure.  value is reported on the SpMV's byte
    model, so it reads as the SpMV's GB/s at that floor."""

    name = "spmv_gather_floor_zipf2_2Mx2M_f32"

    def __init__(self, device, seed=1):
        super().__init__(device, seed)
        from flagsparse_b200 import _native as nat

        self.nat = nat
        self.out = self.torch.empty(148 * 8, dtype=self.torch.float64, device=device)

    def step(self):
        nat = self.nat
        nat.check(nat.lib().fsb_spmv_gather_floor(nat.dtype_code(self.data.dtype), nat.ptr(self.data),
                                                  nat.ptr(self.indices), 0, self.nnz, nat.ptr(self.x),
                                                  nat.ptr(self.out), self.out.numel(),
                                                  nat.stream_of(self.data.device)),
                  "fsb_spmv_gather_floor")

    def e2e_step(self):
        self.x_dev2.copy_(self.x_host, non_blocking=True)
        self.step()

    def e2e_bytes(self):
        return self.K * 4, 0

    def launches_per_step(self):
        return 1


class SpmvZipf64(SpmvZipf):
    """The headline matrix as the float64 drop-in: fp64 values, x and y (same pattern, seed 1)."""

    name = "spmv_csr_zipf2_2Mx2M_f64"
    dtype = "f64"

    def __init__(self, device, seed=1):
        super().__init__(device, seed)
        torch = self.torch
        self.data = self.data.double()
        self.x = self.x.double()
        self.prepared = self.fs.prepare_spmv_csr(self.data, self.indices, self.indptr, self.host["shape"])
        self.y = torch.empty(self.M, dtype=torch.float64, device=device)
        self.x_host = self.x.cpu().pin_memory()
        self.y_host = torch.empty(self.M, dtype=torch.float64).pin_memory()
        self.x_dev2 = torch.empty_like(self.x)
        self.x_buf = [torch.empty_like(self.x) for _ in range(2)]
        self.y_buf = [torch.empty_like(self.y) for _ in range(2)]
        self.y_hosts = [torch.empty(self.M, dtype=torch.float64).pin_memory() for _ in range(2)]

    def config(self):
        return dict(super().config(), workload=self.name, value_dtype="float64")

    def alg_bytes(self):
        return self.nnz * (8 + 4) + (self.M + 1) * 8 + self.K * 8 + self.M * 8

    def e2e_bytes(self):
        return self.K * 8, self.M * 8


class SpmvMtx(SpmvZipf):
    """The SpMV step on a MatrixMarket matrix (fp32 values, int32 columns, x U[-1,1] seed 1)."""

    dtype = "f32"

    def __init__(self, device, path):
        import torch

        import flagsparse_b200 as fs
        from flagsparse_b200 import mtx

        data, indices, indptr, shape = mtx.mtx_to_csr_arrays(path)
        self.name = "spmv_csr_mtx_" + os.path.splitext(os.path.basename(path))[0]
        self.path = path
        x = np.random.default_rng(1).uniform(-1.0, 1.0, shape[1]).astype(np.float32)
        c = {"data": data.astype(np.float32), "indices": indices.astype(np.int32), "indptr": indptr, "x": x,
             "shape": shape}
        self.torch, self.fs, self.host, self.device = torch, fs, c, device
        self.M, self.K = shape
        self.nnz = int(indices.size)
        self.data = torch.from_numpy(c["data"]).to(device)
        self.indices = torch.from_numpy(c["indices"]).to(device)
        self.indptr = torch.from_numpy(indptr).to(device)
        self.x = torch.from_numpy(x).to(device)
        self.prepared = fs.prepare_spmv_csr(self.data, self.indices, self.indptr, shape)
        self.y = torch.empty(self.M, dtype=torch.float32, device=device)
        self.x_host = torch.from_numpy(x).pin_memory()
        self.y_host = torch.empty(self.M, dtype=torch.float32).pin_memory()
        self.x_dev2 = torch.empty_like(self.x)
        self.x_buf = [torch.empty_like(self.x) for _ in range(2)]
        self.y_buf = [torch.empty_like(self.y) for _ in range(2)]
        self.y_hosts = [torch.empty(self.M, dtype=torch.float32).pin_memory() for _ in range(2)]
        self.s_in = torch.cuda.Stream(device=device)
        self.s_out = torch.cuda.Stream(device=device)

    def config(self):
        return {"workload": self.name, "file": os.path.basename(self.path), "rows": self.M, "cols": self.K,
                "nnz": self.nnz, "index_dtype": "int32", "indptr_dtype": "int64",
                "l2": "flushed between timed steps (256 MiB write, then a 50 us device spin that covers the host call)"}


# A device-side spin (~50 us at 1965 MHz) queued after the L2 flush and before a
# step's start event: while the GPU spins, the host finishes the step's Python
# call, so the event pair times the step's kernels and not the host's enqueue.
# The end-to-end leg keeps the host path inside its timed region.
HOST_COVER_CYCLES = 100_000


def _event_median_ms(torch, fn, flush, reps=10, warm=3):
    """Median CUDA-event time of fn() with L2 flushed before every timed call."""
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for i in range(reps):
        flush.fill_(float(i))
        torch.cuda._sleep(HOST_COVER_CYCLES)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        ts.append(s.elapsed_time(e))
    return statistics.median(ts)


def _sampled_rows(torch, c, n_sample, seed):
    """n_sample random rows of c, the positions of their nonzeros, and each position's sample index."""
    rng = np.random.Generator(np.random.PCG64(seed))
    rows = np.sort(rng.choice(c["shape"][0], n_sample, replace=False))
    ptr = c["indptr"]
    take = np.concatenate([np.arange(ptr[r], ptr[r + 1]) for r in rows])
    lens = np.diff(ptr)[rows]
    owner = np.repeat(np.arange(rows.size), lens)
    return rows, take, owner


def _rows_fp64(torch, c, vals64, dense64, rows, take, owner):
    """rows of A @ dense in float64 on the GPU (index_add over the sampled rows' nonzeros)."""
    dev = dense64.device
    cols = torch.from_numpy(c["indices"][take].astype(np.int64)).to(dev)
    v = vals64[torch.from_numpy(take).to(dev)]
    out = torch.zeros(rows.size, dense64.shape[1], dtype=torch.float64, device=dev)
    out.index_add_(0, torch.from_numpy(owner).to(dev), v[:, None] * dense64[cols])
    return out


def _max_rel(got, ref):
    return float((got.detach() - ref).abs().max() / ref.abs().max().clamp_min(1e-300))


class SpmmPowerLaw:
    """C = A B on the 1,000,000 x 1,000,000 power-law matrix (mean 29.7 per row, seed 2).

    Bytes per step, gather model: nnz*(s_v+4) + (M+1)*8 + nnz*N*s + M*N*s (every
    nonzero reads its B row; B exceeds L2).  The compulsory model (B once) is
    reported beside it.
    """

    def __init__(self, device, dname="f32", n=128):
        import torch

        import flagsparse_b200 as fs
        from flagsparse_b200 import workloads
        from flagsparse_b200.sparse_operations import _csr

        self.torch, self.fs, self._csr = torch, fs, _csr
        self.dtype = dname
        self.name = f"spmm_csr_powerlaw_1Mx1M_{dname}_N{n}"
        dt = {"f32": torch.float32, "bf16": torch.bfloat16}[dname]
        c = workloads.zipf_csr(n=1_000_000, scale=32.0 / workloads.ZIPF_MEAN_UNSCALED, seed=2, dtype=np.float32,
                               values="normal")
        self.host = c
        self.M = self.K = c["shape"][0]
        self.n = n
        self.nnz = int(c["indices"].size)
        self.vals = torch.from_numpy(c["data"]).to(device).to(dt)
        self.ind = torch.from_numpy(c["indices"]).to(device)
        self.ptr = torch.from_numpy(c["indptr"]).to(device)
        g = torch.Generator(device=device).manual_seed(2)
        self.B = torch.randn(self.K, n, device=device, generator=g).to(dt)
        self.plan = _csr.SpmmPlan(self.ptr, self.M, dt)
        self.C = torch.empty(self.M, n, dtype=dt, device=device)
        self.route = fs.prepare_spmm_csr_route(self.vals, self.ind, self.ptr, c["shape"])
        self.B_host = self.B.cpu().pin_memory()
        self.C_host = torch.empty(self.M, n, dtype=dt).pin_memory()
        self.B_dev2 = torch.empty_like(self.B)
        self.s = self.B.element_size()

    def config(self):
        return {"workload": self.name, "rows": self.M, "cols": self.K, "nnz": self.nnz, "dense_cols": self.n,
                "seed": 2, "l2": "flushed between timed steps (256 MiB write, then a 50 us device spin that covers the host call)"}

    def alg_bytes(self):
        s = self.s
        return self.nnz * (s + 4) + (self.M + 1) * 8 + self.nnz * self.n * s + self.M * self.n * s

    def compulsory_bytes(self):
        s = self.s
        return self.nnz * (s + 4) + self.K * self.n * s + self.M * self.n * s

    def step(self):
        self._csr.spmm(self.vals, self.ind, self.ptr, self.M, self.K, self.B, self.plan, self.C)

    def e2e_step(self):
        self.B_dev2.copy_(self.B_host, non_blocking=True)
        C = self.fs.flagsparse_spmm_csr_run(self.route, self.B_dev2)
        self.C_host.copy_(C, non_blocking=True)

    def e2e_bytes(self):
        return self.K * self.n * self.s, self.M * self.n * self.s

    def max_rel_err(self, rows, take, owner):
        torch = self.torch
        ref = _rows_fp64(torch, self.host, self.vals.double(), self.B.double(), rows, take, owner)
        return _max_rel(self.C[torch.from_numpy(rows).to(self.C.device)].double(), ref)


class SpmmGatherTma(SpmmPowerLaw):
    """The B-row gather floor of the same SpMM through TMA (fsb_spmm_gather_floor_tma):
    every nonzero's B row copied by tile::gather4 into per-warp shared-memory rings and
    summed, with no row structure (3 CTAs of 4 warps per SM).  value is reported on the
    SpMM's byte model, so it reads as the SpMM's GB/s if its B rows moved that way."""

    def __init__(self, device, dname="f32", n=128):
        super().__init__(device, dname, n)
        from flagsparse_b200 import _native as nat

        self.nat = nat
        self.name = f"spmm_gather_tma_powerlaw_1Mx1M_{dname}_N{n}"
        self.out = self.torch.zeros(148 * 3 * 4, n, dtype=self.torch.float32, device=device)
        self.err = self.torch.zeros(1, dtype=self.torch.int32, device=device)

    def step(self):
        nat = self.nat
        nat.check(nat.lib().fsb_spmm_gather_floor_tma(nat.dtype_code(self.vals.dtype), nat.ptr(self.vals),
                                                      nat.ptr(self.ind), self.nnz, nat.ptr(self.B), self.K,
                                                      int(self.B.stride(0)), self.n, nat.ptr(self.out),
                                                      self.out.shape[0], nat.ptr(self.err),
                                                      nat.stream_of(self.B.device)),
                  "fsb_spmm_gather_floor_tma")

    def e2e_step(self):
        self.B_dev2.copy_(self.B_host, non_blocking=True)
        self.step()

    def e2e_bytes(self):
        return self.K * self.n * self.s, 0

    def launches_per_step(self):
        return 1

    def max_rel_err(self, rows, take, owner):
        return None


class AutogradChungLu:
    """Y = A X forward and dX = A^T dY, dvals = SDDMM(dY, X) backward on the 500,000-node
    Chung-Lu graph (mean degree 25, seed 3), 128 features.

    Bytes per step, gather model: the forward SpMM
    nnz*(s_v+4) + (n+1)*8 + nnz*128*s + n*128*s, and the one-launch backward
    nnz*(4+s_v+4) + (n+1)*8 + nnz*128*s + 2*n*128*s + nnz*s (permutation,
    values through it, columns, row pointers, one dY gather per nonzero, X
    and dX rows, dvals).  The SDDMM alone: 2*nnz*128*s + nnz*(4+4) + nnz*s.
    """

    def __init__(self, device, dname="bf16", part="fwd_bwd"):
        import torch

        import flagsparse_b200 as fs
        from flagsparse_b200 import workloads
        from flagsparse_b200.sparse_operations import sddmm_csr as dm

        self.torch, self.fs, self.dm = torch, fs, dm
        self.dtype = dname
        self.part = part
        self.name = f"autograd_spmm_chung_lu_500k_K128_{dname}" if part == "fwd_bwd" else \
            f"sddmm_csr_chung_lu_500k_K128_{dname}"
        dt = {"f32": torch.float32, "bf16": torch.bfloat16}[dname]
        g = workloads.chung_lu_graph()
        self.host = g
        self.n = g["shape"][0]
        self.nnz = int(g["indices"].size)
        self.ind = torch.from_numpy(g["indices"]).to(device)
        self.ptr = torch.from_numpy(g["indptr"]).to(device)
        gen = torch.Generator(device=device).manual_seed(3)
        self.vals = torch.from_numpy(g["data"]).to(device).to(dt).requires_grad_(True)
        self.X = torch.randn(self.n, 128, device=device, generator=gen).to(dt).requires_grad_(True)
        self.dY = torch.randn(self.n, 128, device=device, generator=gen).to(dt)
        self.p = fs.prepare_spmm_csr_autograd(self.vals.detach(), self.ind, self.ptr, g["shape"])
        self.out = torch.empty(self.nnz, dtype=dt, device=device)
        self.s = self.X.element_size()
        self.X_host = self.X.detach().cpu().pin_memory()
        self.dY_host = self.dY.cpu().pin_memory()
        self.g_host = torch.empty(self.nnz, dtype=dt).pin_memory()

    def config(self):
        return {"workload": self.name, "nodes": self.n, "nnz": self.nnz, "features": 128, "seed": 3,
                "l2": "flushed between timed steps (256 MiB write, then a 50 us device spin that covers the host call)"}

    def alg_bytes(self):
        s, n, z = self.s, self.n, self.nnz
        spmm = z * (s + 4) + (n + 1) * 8 + z * 128 * s + n * 128 * s
        sddmm = 2 * z * 128 * s + z * 8 + z * s
        bwd = z * (4 + s + 4) + (n + 1) * 8 + z * 128 * s + 2 * n * 128 * s + z * s
        return sddmm if self.part == "sddmm" else spmm + bwd

    def step(self):
        if self.part == "sddmm":
            self.dm._native_sddmm(self.p.row_ids, self.p.indices, self.dY, self.X.detach(), None, 1.0, 0.0, self.out)
            return
        self.vals.grad = None
        self.X.grad = None
        self.fs.flagsparse_spmm_csr_autograd(self.vals, self.X, prepared=self.p).backward(self.dY)

    def e2e_step(self):
        with self.torch.no_grad():
            self.X.copy_(self.X_host, non_blocking=True)
            self.dY.copy_(self.dY_host, non_blocking=True)
        self.step()
        grad = self.out if self.part == "sddmm" else self.vals.grad
        self.g_host.copy_(grad, non_blocking=True)

    def e2e_bytes(self):
        return 2 * self.n * 128 * self.s, self.nnz * self.s

    def max_rel_errs(self, rows, take, owner):
        torch = self.torch
        dev = self.X.device
        self.vals.grad = None
        self.X.grad = None
        Y = self.fs.flagsparse_spmm_csr_autograd(self.vals, self.X, prepared=self.p)
        Y.backward(self.dY)
        sel = torch.from_numpy(rows).to(dev)
        v64 = self.vals.detach().double()
        g = self.host
        # the graph and its values are symmetric, so rows of A^T equal rows of A
        err_y = _max_rel(Y[sel].double(), _rows_fp64(torch, g, v64, self.X.detach().double(), rows, take, owner))
        err_dx = _max_rel(self.X.grad[sel].double(), _rows_fp64(torch, g, v64, self.dY.double(), rows, take, owner))
        tk = torch.from_numpy(take).to(dev)
        r_ = torch.from_numpy(rows[owner].astype(np.int64)).to(dev)
        c_ = torch.from_numpy(g["indices"][take].astype(np.int64)).to(dev)
        dv_ref = (self.dY.double()[r_] * self.X.detach().double()[c_]).sum(1)
        err_dv = _max_rel(self.vals.grad[tk].double(), dv_ref)
        return {"max_rel_err_Y": err_y, "max_rel_err_dX": err_dx, "max_rel_err_dvals": err_dv}


class Bsr16:
    """C = A B for the 16 x 16-block BSR matrix: 65,536 x 65,536 blocks (M = K = 1,048,576),
    8 random distinct block columns per block row, bf16 values and B (N = 128), fp32
    accumulation on the tensor cores (seed 2).

    Bytes per step: nnzb*(512 + 4) + (n_brows+1)*8 + nnzb*16*N*2 (one B slab per
    block) + M*N*2.  FLOPs per step: 2 * nnzb * 256 * N.
    """

    def __init__(self, device, n=128):
        import torch

        import flagsparse_b200 as fs
        from flagsparse_b200 import workloads

        self.torch, self.fs = torch, fs
        self.dtype = "bf16"
        self.name = f"bsr16_spmm_65536x65536_blocks_bf16_N{n}"
        c = workloads.bsr16()
        self.n_brows = c["block_shape"][0]
        self.M = self.n_brows * 16
        self.n = n
        self.nnzb = int(c["indices"].size)
        blocks = torch.from_numpy(c["blocks"]).to(device).to(torch.bfloat16)
        self.p = fs.prepare_spmm_bsr16(blocks, torch.from_numpy(c["indices"]).to(device),
                                       torch.from_numpy(c["indptr"]).to(device), (self.M, self.M))
        g = torch.Generator(device=device).manual_seed(2)
        self.B = torch.randn(self.M, n, device=device, generator=g).bfloat16()
        self.C = torch.empty(self.M, n, dtype=torch.bfloat16, device=device)
        self.B_host = self.B.cpu().pin_memory()
        self.C_host = torch.empty(self.M, n, dtype=torch.bfloat16).pin_memory()
        self.B_dev2 = torch.empty_like(self.B)

    def config(self):
        return {"workload": self.name, "block_rows": self.n_brows, "blocks_per_row": 8, "nnzb": self.nnzb,
                "dense_cols": self.n, "seed": 2, "l2": "flushed between timed steps (256 MiB write, then a 50 us device spin that covers the host call)"}

    def alg_bytes(self):
        return self.nnzb * (512 + 4) + (self.n_brows + 1) * 8 + self.nnzb * 16 * self.n * 2 + self.M * self.n * 2

    def flops(self):
        return 2 * self.nnzb * 256 * self.n

    def step(self):
        self.fs.flagsparse_spmm_bsr16(B=self.B, prepared=self.p, out=self.C)

    def e2e_step(self):
        self.B_dev2.copy_(self.B_host, non_blocking=True)
        self.fs.flagsparse_spmm_bsr16(B=self.B_dev2, prepared=self.p, out=self.C)
        self.C_host.copy_(self.C, non_blocking=True)

    def e2e_bytes(self):
        return self.M * self.n * 2, self.M * self.n * 2


class BsrSpmv:
    """y = A x for the 16 x 16-block BSR pattern of Bsr16 (65,536 x 65,536 blocks, 8 per block
    row, seed 2) with fp32 values and x U[-1,1]: FlagSparse's BSR SpMV dtype (spmv_bsr.py:23-28).

    Bytes per step: nnzb*256*4 + nnzb*4 + (n_brows+1)*8 + 2 * M*4 (x and y once).
    """

    dtype = "f32"

    def __init__(self, device):
        import torch

        import flagsparse_b200 as fs
        from flagsparse_b200 import workloads

        self.torch, self.fs = torch, fs
        self.name = "bsr16_spmv_65536x65536_blocks_f32"
        c = workloads.bsr16()
        self.n_brows = c["block_shape"][0]
        self.M = self.n_brows * 16
        self.nnzb = int(c["indices"].size)
        blocks = torch.from_numpy(c["blocks"]).to(device)
        self.p = fs.prepare_spmv_bsr(blocks, torch.from_numpy(c["indices"]).to(device),
                                     torch.from_numpy(c["indptr"]).to(device), (self.M, self.M), 16)
        g = torch.Generator(device=device).manual_seed(2)
        self.x = torch.rand(self.M, device=device, generator=g) * 2 - 1
        self.y = torch.empty(self.M, device=device)
        self.x_host = self.x.cpu().pin_memory()
        self.y_host = torch.empty(self.M).pin_memory()
        self.x_dev2 = torch.empty_like(self.x)

    def config(self):
        return {"workload": self.name, "block_rows": self.n_brows, "blocks_per_row": 8, "nnzb": self.nnzb,
                "block_dim": 16, "seed": 2, "l2": "flushed between timed steps (256 MiB write, then a 50 us device spin that covers the host call)"}

    def alg_bytes(self):
        return self.nnzb * (256 * 4 + 4) + (self.n_brows + 1) * 8 + 2 * self.M * 4

    def step(self):
        self.fs.flagsparse_spmv_bsr(x=self.x, prepared=self.p, out=self.y)

    def e2e_step(self):
        self.x_dev2.copy_(self.x_host, non_blocking=True)
        self.fs.flagsparse_spmv_bsr(x=self.x_dev2, prepared=self.p, out=self.y)
        self.y_host.copy_(self.y, non_blocking=True)

    def e2e_bytes(self):
        return self.M * 4, self.M * 4


class BatchedMix:
    """256 CSR matrices, row counts log-uniform in [1,000, 200,000]: even ids 5-point stencils,
    odd ids random with Poisson(24) rows; fp32, each with x and a 16-column B (seed 4).
    A step is one CUDA-graph replay holding one SpMV and one SpMM over all 256 matrices
    (block-diagonal combined plan, parameters chosen by the batch autotuner).

    Bytes per step: the SpMV formula summed over matrices plus the SpMM compulsory model
    (each B is at most 12.8 MB and stays in L2): sum nnz*(4+4)*2 + (rows+count)*8 + cols*4 +
    rows*4 + cols*16*4 + rows*16*4.
    """

    def __init__(self, device, count=256):
        import torch

        import flagsparse_b200 as fs
        from flagsparse_b200 import workloads

        self.torch = torch
        self.dtype = "f32"
        self.name = f"batched_{count}_uneven_f32_spmv_spmm16"
        mats = workloads.batched_mix(count=count)
        dev = [(torch.from_numpy(m["data"]).to(device), torch.from_numpy(m["indices"]).to(device),
                torch.from_numpy(m["indptr"]).to(device), m["shape"]) for m in mats]
        b = fs.BatchedCsr(dev, n_dense=16)
        for i, m in enumerate(mats):
            b.x_view(i).copy_(torch.from_numpy(m["x"]))
            b.B_view(i).copy_(torch.from_numpy(m["B"]))
        self.b = b
        self.tuning = b.tune()
        b.capture()
        self.x_host = b.x.cpu().pin_memory()
        self.B_host = b.B.cpu().pin_memory()
        self.y_host = torch.empty(b.n_rows, dtype=torch.float32).pin_memory()
        self.C_host = torch.empty(b.n_rows, 16, dtype=torch.float32).pin_memory()

    def config(self):
        b = self.b
        return {"workload": self.name, "matrices": b.count, "rows": b.n_rows, "nnz": b.nnz, "dense_cols": 16,
                "seed": 4, "schedule": {"spmv": b.spmv_cfg, "spmm": b.spmm_cfg,
                                        "fused": b.fused,
                                        "spmv_trials": self.tuning["spmv_trials"],
                                        "spmm_trials": self.tuning["spmm_trials"],
                                        "fused_trials": self.tuning.get("fused_trials", [])},
                "launch": ("one CUDA graph holding one kernel: fused SpMM + SpMV over the block-diagonal batch"
                           if b.fused else "one CUDA graph: SpMV + SpMM launches over the block-diagonal batch"),
                "l2": "flushed between timed steps (256 MiB write, then a 50 us device spin that covers the host call)"}

    def alg_bytes(self):
        spmv, spmm_c, _ = self.b.bytes_models()
        return spmv + spmm_c

    def step(self):
        self.b.run()

    def e2e_step(self):
        b = self.b
        b.x.copy_(self.x_host, non_blocking=True)
        b.B.copy_(self.B_host, non_blocking=True)
        b.run()
        self.y_host.copy_(b.y, non_blocking=True)
        self.C_host.copy_(b.C, non_blocking=True)

    def e2e_bytes(self):
        b = self.b
        return (b.n_cols + b.n_cols * 16) * 4, (b.n_rows + b.n_rows * 16) * 4

    def launches_per_step(self):
        if self.b.fused:
            return 1
        p = self.b._spmv_plan_get()
        return int(p.n_block_units > 0) + int(p.n_units > p.n_block_units) + 1


CASES = {
    "gather_floor": lambda d: SpmvGatherFloor(d),
    "batched_f32": lambda d: BatchedMix(d, BATCH_COUNT),
    "bsr16_bf16_N128": lambda d: Bsr16(d, 128),
    "bsr16_bf16_N64": lambda d: Bsr16(d, 64),
    "bsr_spmv_f32_bd16": lambda d: BsrSpmv(d),
    "spmv_f64": lambda d: SpmvZipf64(d),
    "spmm_f32_N64": lambda d: SpmmPowerLaw(d, "f32", 64),
    "spmm_f32_N128": lambda d: SpmmPowerLaw(d, "f32", 128),
    "spmm_bf16_N128": lambda d: SpmmPowerLaw(d, "bf16", 128),
    "spmm_gather_tma_f32_N128": lambda d: SpmmGatherTma(d, "f32", 128),
    "spmm_gather_tma_bf16_N128": lambda d: SpmmGatherTma(d, "bf16", 128),
    "autograd_f32": lambda d: AutogradChungLu(d, "f32"),
    "autograd_bf16": lambda d: AutogradChungLu(d, "bf16"),
    "sddmm_f32_K128": lambda d: AutogradChungLu(d, "f32", part="sddmm"),
    "sddmm_bf16_K128": lambda d: AutogradChungLu(d, "bf16", part="sddmm"),
}


# matrices in the batched case (--batched-count; the headline extras use 256)
BATCH_COUNT = 256

# native kernels per step: the forward SpMM and the one-launch backward
# (dX and dvals from fsb_spmm_csr_backward).
LAUNCHES_PER_STEP = {"autograd_f32": 2, "autograd_bf16": 2}


def measure_extras(torch, device, flush, peak):
    """SpMM on the power-law matrix and the differentiable layer on the Chung-Lu graph:
    CUDA-event medians (L2 flushed) and errors on sampled rows against float64 on the GPU."""
    out = {}
    spmm = {}
    rows = take = owner = None
    for key in ("spmm_f32_N64", "spmm_f32_N128", "spmm_bf16_N128"):
        case = CASES[key](device)
        if rows is None:
            rows, take, owner = _sampled_rows(torch, case.host, 2000, 7)
        ms = _event_median_ms(torch, case.step, flush)
        gather, comp = case.alg_bytes(), case.compulsory_bytes()
        spmm[key[5:]] = {"ms": round(ms, 4), "gather_model_gbs": round(gather / ms / 1e6, 1),
                         "compulsory_model_gbs": round(comp / ms / 1e6, 1),
                         "gather_model_frac": round(gather / ms / 1e6 / peak, 3),
                         "max_rel_err_vs_fp64_sampled": case.max_rel_err(rows, take, owner)}
        nnz, M = case.nnz, case.M
        del case
    out["spmm_powerlaw_1Mx1M"] = dict(spmm, nnz=nnz, rows=M, mean_row=round(nnz / M, 2),
                                      bytes_models="gather: nnz*(s_v+4)+(M+1)*8+nnz*N*s+M*N*s; "
                                                   "compulsory: nnz*(s_v+4)+K*N*s+M*N*s")
    out["spmm_powerlaw_1Mx1M"]["cpu_reference_f32_N128"] = cpu_torch_spmm()
    layer = {}
    rows = None
    for dname in ("f32", "bf16"):
        case = AutogradChungLu(device, dname)
        sd = AutogradChungLu.__new__(AutogradChungLu)
        sd.__dict__.update(case.__dict__)
        sd.part = "sddmm"
        if rows is None:
            rows, take, owner = _sampled_rows(torch, case.host, 500, 9)
        ms = _event_median_ms(torch, case.step, flush)
        ms_sd = _event_median_ms(torch, sd.step, flush)
        layer[dname] = dict({"fwd_bwd_ms": round(ms, 4), "fwd_bwd_gather_model_gbs": round(case.alg_bytes() / ms / 1e6, 1),
                             "sddmm_ms": round(ms_sd, 4)}, **case.max_rel_errs(rows, take, owner))
        nnz = case.nnz
        del case, sd
    layer["bf16_speedup_vs_f32"] = round(layer["f32"]["fwd_bwd_ms"] / layer["bf16"]["fwd_bwd_ms"], 3)
    layer["cpu_reference_f32"] = cpu_torch_autograd()
    out["autograd_chung_lu_500k_K128"] = dict(layer, nnz=nnz, error_reference="float64 on the GPU, 500 sampled rows")
    case = BatchedMix(device, 256)
    ms = _event_median_ms(torch, case.step, flush)
    spmv_b, spmm_c, spmm_g = case.b.bytes_models()
    out["batched_256_uneven_f32"] = {"ms": round(ms, 4), "gbs": round((spmv_b + spmm_c) / ms / 1e6, 1),
                                     "gather_model_gbs": round((spmv_b + spmm_g) / ms / 1e6, 1),
                                     "matrices": case.b.count, "rows": case.b.n_rows, "nnz": case.b.nnz,
                                     "schedule": {"spmv": case.b.spmv_cfg, "spmm": case.b.spmm_cfg},
                                     "launch": ("one CUDA graph replay of one fused SpMM + SpMV kernel over all 256 matrices"
                                                if case.b.fused else
                                                "one CUDA graph replay (SpMV + SpMM over all 256 matrices)")}
    del case
    case = Bsr16(device)
    ms = _event_median_ms(torch, case.step, flush)
    bf16_peak = _measured_bf16_tflops()
    out["bsr16_spmm_bf16_N128"] = {"ms": round(ms, 4), "gbs": round(case.alg_bytes() / ms / 1e6, 1),
                                   "hbm_frac": round(case.alg_bytes() / ms / 1e6 / peak, 3),
                                   "tflops": round(case.flops() / ms / 1e9, 1),
                                   "tensor_frac_of_measured_bf16": round(case.flops() / ms / 1e9 / bf16_peak, 4),
                                   "nnzb": case.nnzb, "bound": "hbm (12 flop/byte, far below the tensor ridge)"}
    del case
    case = SpmvGatherFloor(device)
    ms = _event_median_ms(torch, case.step, flush)
    out["spmv_gather_floor_zipf2M_f32"] = {
        "ms": round(ms, 4), "spmv_model_gbs": round(case.alg_bytes() / ms / 1e6, 1),
        "hbm_frac": round(case.alg_bytes() / ms / 1e6 / peak, 3),
        "what": "sum of data[i]*x[indices[i]] over every nonzero of the headline matrix (no rows): the time "
                "its values, columns and x gathers alone take"}
    del case
    case = SpmvZipf64(device)
    ms = _event_median_ms(torch, case.step, flush)
    out["spmv_f64_zipf2M"] = {"ms": round(ms, 4), "gbs": round(case.alg_bytes() / ms / 1e6, 1),
                              "hbm_frac": round(case.alg_bytes() / ms / 1e6 / peak, 3),
                              "bytes_model": "nnz*(8+4)+(M+1)*8+K*8+M*8"}
    del case
    case = BsrSpmv(device)
    ms = _event_median_ms(torch, case.step, flush)
    out["bsr_spmv_f32_bd16"] = {"ms": round(ms, 4), "gbs": round(case.alg_bytes() / ms / 1e6, 1),
                                "hbm_frac": round(case.alg_bytes() / ms / 1e6 / peak, 3), "nnzb": case.nnzb,
                                "bytes_model": "nnzb*(256*4+4)+(n_brows+1)*8+2*M*4"}
    return out


def cpu_torch_spmm(reps=2):
    """C = A B on the host cores through torch.sparse.mm on a CPU sparse_csr_tensor (the
    reference's CPU path) for the 1M power-law matrix and a 128-column fp32 B."""
    import torch

    from flagsparse_b200 import workloads

    nthreads = os.cpu_count() or 1
    torch.set_num_threads(nthreads)
    c = workloads.zipf_csr(n=1_000_000, scale=32.0 / workloads.ZIPF_MEAN_UNSCALED, seed=2, dtype=np.float32,
                           values="normal")
    A = torch.sparse_csr_tensor(torch.from_numpy(c["indptr"]), torch.from_numpy(c["indices"]),
                                torch.from_numpy(c["data"]), size=c["shape"])
    B = torch.from_numpy(workloads.dense_normal(c["shape"][1], 128, seed=2))
    s_per, n = _wall_per_step(lambda: torch.sparse.mm(A, B), 0.0, max_reps=reps)
    return {"ms": round(s_per * 1e3, 2), "cores": nthreads, "kind": "reference",
            "sample": f"{n} SpMMs through torch.sparse.mm on a CPU sparse_csr_tensor, fp32"}


def cpu_torch_autograd(reps=2):
    """Forward Y = A X and backward (dX, and dA on A's pattern) on the host cores through
    torch's sparse CSR autograd (torch.sparse.mm with A a leaf) on the 500,000-node Chung-Lu
    graph, fp32, K = 128."""
    import torch

    from flagsparse_b200 import workloads

    nthreads = os.cpu_count() or 1
    torch.set_num_threads(nthreads)
    g = workloads.chung_lu_graph()
    n = g["shape"][0]
    X = torch.from_numpy(workloads.dense_normal(n, 128, seed=4)).requires_grad_(True)
    dY = torch.from_numpy(workloads.dense_normal(n, 128, seed=3))
    A = torch.sparse_csr_tensor(torch.from_numpy(g["indptr"]), torch.from_numpy(g["indices"].astype(np.int64)),
                                torch.from_numpy(g["data"]), size=g["shape"], requires_grad=True)

    def step():
        A.grad = None
        X.grad = None
        torch.sparse.mm(A, X).backward(dY)

    s_per, k = _wall_per_step(step, 0.0, max_reps=reps)
    return {"fwd_bwd_ms": round(s_per * 1e3, 2), "cores": nthreads, "kind": "reference",
            "sample": f"{k} forward + backward steps through torch's sparse CSR autograd on the host, fp32"}


def _cpu_measure(make_workload_host, budget_s, nthreads):
    """Repeat the CPU oracle over the whole matrix until ~budget_s seconds; return (s per step, reps)."""
    reps, t0 = 0, time.perf_counter()
    while True:
        make_workload_host(nthreads)
        reps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or reps >= 200:
            return el / reps, reps


# ---------------------------------------------------------------- main

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=12.0, help="seconds of CPU-oracle work for cpu_baseline")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the SpMM and autograd measurements")
    ap.add_argument("--case", default="spmv", choices=["spmv"] + sorted(CASES),
                    help="workload of the timed steps (default: the SpMV headline)")
    ap.add_argument("--mtx", default=None, help="time the SpMV on this MatrixMarket file instead (fp32 values)")
    ap.add_argument("--batched-count", type=int, default=256,
                    help="matrices in --case batched_f32 (a smaller batch for profiling)")
    args = ap.parse_args()
    global BATCH_COUNT
    BATCH_COUNT = args.batched_count
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)

    if args.mtx:
        wl = SpmvMtx(device, args.mtx)
    elif args.case == "spmv" and world > 1:
        wl = SpmvZipfSharded(device, rank, world)
    else:
        wl = SpmvZipf(device) if args.case == "spmv" else CASES[args.case](device)
    headline = args.case == "spmv" and not args.mtx
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        wl.step()
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank)
    sampler.start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    sampler.mark("timed_start")
    for i in range(args.steps):
        flush.fill_(float(i))
        torch.cuda._sleep(HOST_COVER_CYCLES)
        starts[i].record()
        wl.step()
        ends[i].record()
    torch.cuda.synchronize()
    sampler.mark("timed_end")
    barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    t_ms = sum(step_ms)

    # end-to-end through the public API with host buffers
    pipelined = hasattr(wl, "e2e_run") and getattr(wl, "pipelined", True)
    if pipelined:
        wl.e2e_run(2)
    else:
        for _ in range(2):
            wl.e2e_step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record()
    if pipelined:
        wl.e2e_run(args.steps)
    else:
        for _ in range(args.steps):
            wl.e2e_step()
    e1.record()
    torch.cuda.synchronize()
    sampler.mark("phase_end")
    barrier()
    clocks = sampler.stop()
    e2e_ms = e0.elapsed_time(e1)

    if world > 1:
        tt = torch.tensor([t_ms, e2e_ms], dtype=torch.float64, device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_ms, e2e_ms = tt.tolist()

    alg = wl.alg_bytes()
    # a sharded workload splits one fixed job (strong scaling); replicas repeat it per rank (weak)
    job = wl.total_bytes() if hasattr(wl, "total_bytes") else world * alg
    scaling = "strong" if hasattr(wl, "total_bytes") else "weak"
    value = job * args.steps / (t_ms * 1e-3) / 1e9
    e2e_val = job * args.steps / (e2e_ms * 1e-3) / 1e9
    peak, peak_src = _measured_peaks()
    mean_launch_ms = statistics.mean(step_ms)
    achieved = alg / (mean_launch_ms * 1e-3) / 1e9
    traffic = _ncu_traffic(wl.name)
    h2d, d2h = wl.e2e_bytes()

    extras = None
    if world == 1 and headline and not args.no_extras:
        extras = measure_extras(torch, device, flush, peak)

    cpu = cpu_port = None
    if rank == 0 and world == 1 and headline and not args.no_cpu:
        ref = TorchCpuSpmv(wl.host)
        s_per, reps = _wall_per_step(ref.step, args.cpu_budget)
        cpu = {"value": round(alg / s_per / 1e9, 3), "unit": "GB/s", "cores": ref.nthreads, "kind": "reference",
               "sample": f"{reps} full SpMVs of the same matrix through torch.sparse.mm on a CPU sparse_csr_tensor "
                         f"(the reference's CPU path; fp32 values summed in fp64), {s_per * 1e3:.1f} ms each"}
        del ref
        from oracle import oracle

        nthreads = oracle.max_threads()
        s_per, reps = _cpu_measure(wl.cpu_run, args.cpu_budget, nthreads)
        cpu_port = {"value": round(alg / s_per / 1e9, 3), "unit": "GB/s", "cores": nthreads, "kind": "port",
                    "sample": f"{reps} full SpMVs of the same matrix (fp32 values, fp64 row sums), "
                              f"{s_per * 1e3:.1f} ms each, the C restatement, OpenMP over rows"}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": round(value, 2),
            "unit": "GB/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(t_ms / args.steps, 5),
            "higher_is_better": True,
            "scaling": scaling,
            "vs_baseline": None,
            "dtype": wl.dtype,
            "data": ("synthetic (seeded Zipf(2) power-law CSR, values/x U[-1,1])" if headline
                     else f"MatrixMarket file {os.path.basename(args.mtx)}, x U[-1,1]" if args.mtx
                     else "synthetic (seeded generators; see config.workload)"),
            "config": dict(wl.config(), parallelism=(f"rows{world}" if scaling == "strong" else f"replicas{world}")
                           if world > 1 else "single"),
            "e2e": {"value": round(e2e_val, 2), "unit": "GB/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "schedule": ("pipelined: x upload of step i+1 and y download of step i-1 overlap "
                                 "the SpMV of step i (double buffers, three streams)" if pipelined
                                 else "serial: upload, compute, download per step")},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs, copy burst)",
                         "alg_bytes_per_launch": alg},
            "cpu_baseline": cpu,
            "cpu_baseline_port": cpu_port,
            "gpu_launches": args.steps * (wl.launches_per_step() if hasattr(wl, "launches_per_step")
                                          else LAUNCHES_PER_STEP.get(args.case, 1)),
            "clocks": clocks,
            "extras": extras,
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args, rank, world):
    """The reference's CPU path (torch.sparse.mm on a CPU sparse_csr_tensor, fp32 values summed
    in fp64) on the headline matrix with all host threads, rank 0 only; the C restatement of
    the same semantics is timed beside it."""
    if rank != 0:
        return
    from flagsparse_b200 import workloads
    from oracle import oracle

    c = workloads.zipf_csr(n=2_000_000, seed=1, dtype=np.float32)
    nnz = int(c["indices"].size)
    M, K = c["shape"]
    alg = nnz * 8 + (M + 1) * 8 + K * 4 + M * 4
    ref = TorchCpuSpmv(c)
    for _ in range(args.warmup):
        ref.step()
    steps = args.steps
    t0 = time.perf_counter()
    for _ in range(steps):
        ref.step()
    el = time.perf_counter() - t0
    value = alg * steps / el / 1e9
    nthreads = oracle.max_threads()
    port_s, port_reps = _cpu_measure(
        lambda nt: oracle.spmv_f32_acc64(c["indptr"], c["indices"], c["data"], c["x"], nthreads=nt),
        min(args.cpu_budget, 5.0), nthreads)
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": round(el / steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Zipf(2) power-law CSR, values/x U[-1,1])",
        "config": dict(spmv_zipf_config(M, K, nnz), parallelism=f"rows{world}" if world > 1 else "single"),
        "impl": "reference",
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": ref.nthreads, "kind": "reference",
                         "sample": f"{steps} full SpMVs through torch.sparse.mm on a CPU sparse_csr_tensor "
                                   "(the reference's CPU path), fp32 values summed in fp64"},
        "cpu_baseline_port": {"value": round(alg / port_s / 1e9, 3), "unit": "GB/s", "cores": nthreads,
                              "kind": "port", "sample": f"{port_reps} full SpMVs, the C restatement (fp32 values, "
                                                        "fp64 row sums), OpenMP over rows"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
