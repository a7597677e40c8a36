"""One frame split across ranks by node-row bands (2d_aldic_b200/split.py):
world-size-2 and -3 gloo ranks on the CPU, each holding only its band of the
images, run the per-subset work of its band with the CPU restatement,
all-gather the results once per stage and replicate the grid-wide steps.
The split frame must equal the whole-frame oracle (main_ALDIC.m Sections
3-6): the node grid exactly, U and F within 1e-8 px (band-local coordinates
round differently in the last bits)."""
import importlib
import math
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

split = importlib.import_module("2d_aldic_b200.split")


class OracleBackend:
    """The split frame's per-rank arithmetic on the CPU restatement."""

    def __init__(self):
        import oracle
        self.O = oracle

    def roi_sums(self, block):
        b = np.asarray(block).astype(np.int64)
        return int(b.sum()), int((b * b).sum()), int(b.size)

    def load(self, f, g, stats):
        out = []
        for img, (s1, s2, n) in zip((f, g), stats):
            m = s1 / n                       # orc_normalize's statistics of integer images
            sd = math.sqrt((float(s2) - m * float(s1)) / (n - 1))
            out.append(((img.astype(np.float64) - m) / sd, m))
        (self.fn, _), (self.gn, self.mg) = out
        self.f, self.g = np.ascontiguousarray(f), np.ascontiguousarray(g)
        self.dx, self.dy = self.O.gradient(self.fn)

    def search(self, gridx, gridy, w, step, s):
        x, y, u, v, _, _ = self.O.int_search(self.f, self.g, self.mg, gridx, gridy, w, step, (s, s))
        return x, y, u, v

    def icgn(self, coords, U0, w, tol):
        U, F, it, H = self.O.icgn_batch(self.fn, self.gn, self.dx, self.dy, coords, U0, w, tol)
        return U, F, it, np.asarray(H).T

    def subpb1(self, coords, UOld, FOld, vdual, H21, w, mu, tol):
        return self.O.subpb1_batch(self.fn, self.gn, self.dx, self.dy, coords, UOld, FOld, vdual,
                                   np.ascontiguousarray(np.asarray(H21).T), w, mu, tol)

    def inpaint(self, M, N, z):
        return self.O.inpaint_springs(M, N, np.asarray(z))

    def localicgn_post(self, M, N, it, U, F):
        return self.O.localicgn_post(M, N, it, U, F)

    def subpb1_post(self, M, N, it, U):
        return self.O.subpb1_post(M, N, it, U)[0]

    def subpb2(self, M, N, h, beta, mu, U, F, ud, vd):
        return self.O.subpb2(M, N, h, beta, mu, U, F, ud, vd)[0]

    def nodal_strain(self, M, N, h, U):
        return self.O.nodal_strain(M, N, h, U)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    return dist


def _rank_main(rank, world, port, q):
    dist = _init(rank, world, port)
    try:
        synth = importlib.import_module("2d_aldic_b200.synth")
        import oracle
        oracle.set_threads(2)
        wl = synth.workload("plain512", scale_down=2)
        f, g = wl.images()
        ex = split.Exchange()
        r = split.split_frame(OracleBackend(), ex, rank, f, g, wl.winsize, wl.step, wl.search,
                              tol=wl.tol, n_admm=2)
        q.put((rank, r["U"], r["F"], r["x0"], r["y0"], r["band"], r["rows"], ex.calls))
    finally:
        dist.destroy_process_group()


def _rank_main_gpu(rank, world, port, q):
    dist = _init(rank, world, port)
    try:
        aldic = importlib.import_module("2d_aldic_b200")
        synth = importlib.import_module("2d_aldic_b200.synth")
        wl = synth.workload("plain512", scale_down=2)
        f, g = wl.images()
        be = split.DeviceBackend(0, precision=aldic.FP64)
        r = split.split_frame(be, split.Exchange(), rank, f, g, wl.winsize, wl.step, wl.search,
                              tol=wl.tol, n_admm=2)
        be.close()
        q.put((rank, r["U"], r["F"], r["x0"], r["y0"], r["band"], r["rows"], 0))
    finally:
        dist.destroy_process_group()


def _run(target, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = [q.get(timeout=600) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def _whole(oracle, synth):
    wl = synth.workload("plain512", scale_down=2)
    f, g = wl.images()
    return f, oracle.frame(f, g, wl.winsize, wl.step, wl.search, tol=wl.tol, n_admm=2)


@pytest.mark.parametrize("world", [2, 3])
def test_split_frame_equals_whole_frame(oracle, synth, world):
    res = _run(_rank_main, world)
    f, ro = _whole(oracle, synth)
    H = f.shape[0]
    bands = sorted((r[5], r[6]) for r in res)
    assert bands[0][0][0] == 0 and bands[-1][0][1] == ro["N"]
    for (_, rows) in bands:
        assert rows[1] - rows[0] < H                      # no rank holds the whole image
    for rank, U, F, x0, y0, band, rows, calls in res:
        np.testing.assert_array_equal(x0, ro["x0"])
        np.testing.assert_array_equal(y0, ro["y0"])
        assert np.abs(U - ro["U"]).max() < 1e-8
        assert np.abs(F - ro["F"]).max() < 1e-8
        # ROI sums (2), search, LocalICGN, one per ADMM step
        assert calls == 2 + 1 + 1 + 2


@pytest.mark.gpu
@pytest.mark.parametrize("world", [1, 2])
def test_split_frame_on_device_matches_oracle(oracle, synth, world):
    """The same split frame with every rank's per-subset work and replicated
    steps on the GPU through the C ABI (band images in each rank's own
    context, the summed ROI statistics set with aldic_set_stats); the ranks
    exchange over gloo and share the one GPU of the test box (no kernel of
    one rank waits on another's).  FP64: within 1e-4 px of the whole-frame
    oracle."""
    res = _run(_rank_main_gpu, world)
    f, ro = _whole(oracle, synth)
    for rank, U, F, x0, y0, band, rows, _ in res:
        np.testing.assert_array_equal(x0, ro["x0"])
        assert np.abs(U - ro["U"]).max() < 1e-4
