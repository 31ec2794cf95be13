"""Single domain decomposed into x slabs (resistivemhd_gpu_b200/slab.py over
the C ABI's rmhd2d_create_slab / rmhd2d_slab_*), which replaces the
multi-GPU library's decomposition (ResistiveMHD_multiGPU_cuda/
ResistiveMHD2D_GPU/mpi.cu:104-276, resistiveMHD2D.cu:550,574): after any
number of steps the slabs hold, bit for bit, what one solver on the whole
domain holds -- the oracle's states and dts.

On the CPU the slabs run on the host build of the whole C ABI
(tests/host_build.py): in one process (SlabGroup), and as 2 and 3 gloo ranks
in spawned processes (SlabDomain over torch.distributed point-to-point and
all-reduce).  On the GPU the CUDA library runs SlabGroup and a one-rank
SlabDomain over NCCL."""
import ctypes
import dataclasses
import datetime
import os
import socket

import numpy as np
import pytest

from host_build import build_host_abi, has_fma

# (x walls, y walls, eta table, interior shape, slabs, steps)
CASES = [
    ("periodic", "periodic", True, (30, 14), 3, 5),
    ("symmetric", "symmetric", False, (25, 16), 2, 5),
    ("periodic", "symmetric", True, (19, 13), 2, 5),    # the domain's ghost column 0 in the first slab's halo
    ("flare", "wall", False, (22, 12), 3, 4),
    ("zero_gradient", "periodic", True, (27, 17), 4, 4),
    ("periodic", "symmetric", False, (12, 10), 1, 4),   # one slab whose halos are its own far edges
]


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _setup(bcx, bcy, table, shape, seed=17):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*shape, seed=seed, bc=bcx, with_table=table)
    return dataclasses.replace(s, bc=bcx, bc_y=bcy)


def test_partition():
    from resistivemhd_gpu_b200.slab import partition

    assert partition(20, 3) == [(0, 7), (7, 7), (14, 6)]
    assert partition(9, 1) == [(0, 9)]
    with pytest.raises(ValueError):
        partition(17, 3)                 # a slab owns at least 6 columns, a solver's smallest interior


@pytest.fixture(scope="module")
def host_abi_path(tmp_path_factory):
    if not has_fma():
        pytest.skip("the host has no fused multiply-add to model the device build with")
    d = tmp_path_factory.mktemp("slabhost")
    build_host_abi(d)
    return d / "librmhd2d_host.so"


def _bind(path):
    """The Python mirror bound to the host build of the C ABI."""
    from resistivemhd_gpu_b200 import _lib

    lib = ctypes.CDLL(str(path))
    for name, res, args in _lib.SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib._lib = lib
    return lib


@pytest.mark.parametrize("bcx,bcy,table,shape,parts,steps", CASES)
def test_slab_group_equals_oracle_on_host_build(host_abi_path, oracle, monkeypatch, bcx, bcy, table, shape, parts,
                                                steps):
    from resistivemhd_gpu_b200 import _lib
    from resistivemhd_gpu_b200.slab import SlabGroup

    monkeypatch.setattr(_lib, "_lib", None)
    _bind(host_abi_path)
    s = _setup(bcx, bcy, table, shape)
    want, want_dts, crashed = oracle.run(s, s.state, steps)
    assert crashed == -1
    with SlabGroup(s, parts, torch_device="cpu") as g:
        dts = []
        for _ in range(steps):
            g.step()
            dts.append(g.dt)
        assert _bits(np.array(dts)).tolist() == _bits(want_dts).tolist()
        assert np.array_equal(_bits(g.get_state()), _bits(want))
        assert not g.check_crashed()


def test_slab_refusals_on_host_build(host_abi_path, monkeypatch):
    from resistivemhd_gpu_b200 import _lib
    from resistivemhd_gpu_b200.slab import SlabGroup

    monkeypatch.setattr(_lib, "_lib", None)
    _bind(host_abi_path)
    s = _setup("periodic", "periodic", False, (12, 10))
    with SlabGroup(s, 2, torch_device="cpu") as g:
        sol = g.slabs[0].solver
        for call in (sol.step, lambda: sol.run(2), sol.calculate_dt, sol.apply_boundary,
                     lambda: sol.set_state(s.state[:sol.nx], apply_boundary=True), lambda: sol.adjoint_forward(2)):
            with pytest.raises(_lib.RMHDError) as e:
                call()
            assert e.value.status == 4                  # RMHD2D_ERR_STATE
    from resistivemhd_gpu_b200 import Solver

    lib = _lib.load()
    cfg = Solver.make_config(12, 12, 0.1, 0.1)
    h = ctypes.c_void_p()
    assert lib.rmhd2d_create_slab(ctypes.byref(cfg), 2, ctypes.byref(h)) == 1   # low wall without the origin flag
    cfg.ct_scheme = 1
    assert lib.rmhd2d_create_slab(ctypes.byref(cfg), 7, ctypes.byref(h)) == 1   # CT-Contact


def _free_port() -> int:
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_worker(rank, world, port, lib_path, case, out):
    import sys

    import torch.distributed as dist

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, here)
    _bind(lib_path)
    from resistivemhd_gpu_b200.slab import SlabDomain

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        bcx, bcy, table, shape, steps = case
        dom = SlabDomain(_setup(bcx, bcy, table, shape), torch_device="cpu")
        dts = []
        for _ in range(steps):
            dom.step()
            dts.append(dom.dt)
        out.put((rank, dom.columns, dom.get_state(), dts, dom.check_crashed()))
        dom.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,case", [
    (2, ("periodic", "symmetric", True, (17, 12), 4)),
    (3, ("symmetric", "periodic", False, (20, 11), 4)),
    (2, ("periodic", "periodic", False, (12, 9), 3)),
])
def test_slab_domain_on_gloo_ranks_equals_oracle(host_abi_path, oracle, world, case):
    """Each rank a spawned process with its slab of the domain; halos move by
    gloo send/recv, the words by an all-reduce.  Every rank's own columns
    and dts equal the oracle's whole-domain run."""
    import torch.multiprocessing as mp

    bcx, bcy, table, shape, steps = case
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_worker, args=(r, world, port, str(host_abi_path), case, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted((q.get(timeout=300) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    s = _setup(bcx, bcy, table, shape)
    want, want_dts, _ = oracle.run(s, s.state, steps)
    covered = 0
    for rank, (x0, n), local, dts, crashed in results:
        assert not crashed
        assert _bits(np.array(dts)).tolist() == _bits(want_dts).tolist()
        assert np.array_equal(_bits(local[3:3 + n]), _bits(want[3 + x0:3 + x0 + n]))
        covered += n
    assert covered == s.nx - 6


@pytest.mark.gpu
@pytest.mark.parametrize("bcx,bcy,table,shape,parts,steps", CASES + [("symmetric", "symmetric", True, (333, 130), 4, 6)])
def test_slab_group_equals_whole_domain_on_gpu(gpu, bcx, bcy, table, shape, parts, steps):
    from resistivemhd_gpu_b200 import Solver
    from resistivemhd_gpu_b200.slab import SlabGroup

    s = _setup(bcx, bcy, table, shape)
    with Solver.from_setup(s, precision="fp64_exact") as whole:
        dts = []
        for _ in range(steps):
            whole.step()
            dts.append(whole.dt)
        want = whole.get_state()
    with SlabGroup(s, parts) as g:
        got_dts = []
        for _ in range(steps):
            g.step()
            got_dts.append(g.dt)
        assert _bits(np.array(got_dts)).tolist() == _bits(np.array(dts)).tolist()
        assert np.array_equal(_bits(g.get_state()), _bits(want))


@pytest.mark.gpu
@pytest.mark.parametrize("bcx,bcy", [("symmetric", None), ("periodic", "symmetric")])
def test_slab_group_full_size_harris_on_gpu(gpu, bcx, bcy):
    """The headline workload, the Harris sheet on 2048x1024 cells with its eta
    table (its symmetric walls, and periodic in x), in 4 slabs of 512
    columns: 10 steps bit for bit those of one solver on the whole domain."""
    from resistivemhd_gpu_b200 import Solver, setups
    from resistivemhd_gpu_b200.slab import SlabGroup

    s = dataclasses.replace(setups.harris_sheet(2048, 1024), bc=bcx, bc_y=bcy)
    steps = 10
    with Solver.from_setup(s, precision="fp64_exact") as whole:
        dts = []
        for _ in range(steps):
            whole.step()
            dts.append(whole.dt)
        want = whole.get_state()
    with SlabGroup(s, 4) as g:
        assert [sl.n for sl in g.slabs] == [512] * 4
        got_dts = []
        for _ in range(steps):
            g.step()
            got_dts.append(g.dt)
        assert _bits(np.array(got_dts)).tolist() == _bits(np.array(dts)).tolist()
        assert np.array_equal(_bits(g.get_state()), _bits(want))
        assert not g.check_crashed()


@pytest.mark.gpu
def test_slab_domain_one_nccl_rank_on_gpu(gpu, oracle):
    """SlabDomain over an NCCL process group of one rank (periodic x: the
    slab's halos are its own far edges; the words' all-reduce runs)."""
    import torch
    import torch.distributed as dist

    from resistivemhd_gpu_b200.slab import SlabDomain

    s = _setup("periodic", "symmetric", True, (40, 24))
    want, want_dts, _ = oracle.run(s, s.state, 5)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ["MASTER_PORT"] = str(_free_port())
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        dom = SlabDomain(s)
        dom.run(5)
        assert dom.dt == want_dts[-1]
        assert np.array_equal(_bits(dom.get_state()), _bits(want))
        dom.close()
    finally:
        dist.destroy_process_group()
