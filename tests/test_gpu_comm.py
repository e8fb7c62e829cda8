"""The NCCL exchange through the C ABI (n2w_comm_*) on one GPU: a one-rank
communicator is the identity for every all-reduce, the barrier returns, and
data-parallel training with it (n2w_nc_train_dp) is n2w_nc_train bit for bit.
Several ranks need several GPUs, which these runs do not have; the ranks'
host logic is covered by tests/test_shard.py with gloo."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def comm(gpu):
    from n2w.shard import NcclComm

    c = NcclComm(0, 1, key=f"test_{os.getpid()}")
    yield c
    c.close()


def test_one_rank_allreduce_is_identity(gpu, comm):
    from n2w._lib import N2W_DTYPE_F32, N2W_OP_MAX, N2W_OP_SUM, call

    x = np.random.default_rng(1).normal(size=1000)
    for op in ("sum", "max", "min"):
        np.testing.assert_array_equal(comm.allreduce_host([x], op)[0], x)
    f = np.arange(17, dtype=np.float32)
    d_in, d_out = gpu.DeviceBuffer.from_array(f), gpu.DeviceBuffer(f.nbytes)
    for op in (N2W_OP_SUM, N2W_OP_MAX):
        call("n2w_comm_allreduce", comm.h, d_in.ptr, d_out.ptr, len(f), N2W_DTYPE_F32, op, None)
        np.testing.assert_array_equal(d_out.download(np.float32), f)
    comm.barrier()
    rank, world = C.c_int(), C.c_int()
    call("n2w_comm_info", comm.h, C.byref(rank), C.byref(world))
    assert (rank.value, world.value) == (0, 1)


def test_point_stats_allreduce_identity(gpu, comm):
    m = gpu.Mesh.bumpy_sphere_trig(32, 64, 0.08, 6, 8)
    m.normalize()
    bvh = gpu.Bvh(m, 4, "sah")
    pts = np.array([[0.1, 0.2, -0.1], [-0.3, 0.1, 0.25]], np.float32)
    st = gpu.PointStatsBuffers.allocate(len(pts))
    gpu.wos_estimate(bvh, gpu.problem_charges_seeded(8, 1.6, 2.0, 12345), pts,
                     options=gpu.walk_options(walks_per_point=256, seed=3), stats=st)
    before = st.download()
    comm.allreduce_point_stats_device(st, len(pts))
    after = st.download()
    for k in ("sum", "sum_sq", "count", "mean_steps", "forced"):
        np.testing.assert_array_equal(before[k], after[k])


def test_data_parallel_training_one_rank_equals_single_process(gpu, comm):
    """n2w_nc_train_dp on a one-rank communicator runs what n2w_nc_train runs.
    Training is not bit-reproducible: the interior sampler hands out its
    accepted points in atomic order and the hash-grid gradient is a float
    atomic scatter, so two plain runs already differ.  The data-parallel run
    must differ from a plain run no more than a second plain run does, in the
    loss curve and in the parameters."""
    from n2w import nc
    from n2w._lib import call

    m = gpu.Mesh.bumpy_sphere_trig(32, 64, 0.08, 6, 8)
    m.normalize()
    bvh = gpu.Bvh(m, 4, "sah")
    p = gpu.problem_charges_seeded(8, 1.6, 2.0, 12345)
    cfg = gpu.cache_config(n_levels=8, log2_hashmap_size=14, max_resolution=256.0)
    o = nc.train_options(m, steps=5, batch=4096, walks_per_label=8)

    def run(dp):
        c = gpu.Cache(cfg)
        losses = np.zeros(5, np.float32)
        if dp:
            call("n2w_nc_train_dp", c.handle, bvh.handle, C.byref(p), C.byref(o), comm.h,
                 C.c_void_p(losses.ctypes.data), None)
        else:
            call("n2w_nc_train", c.handle, bvh.handle, C.byref(p), C.byref(o), C.c_void_p(losses.ctypes.data),
                 None)
        return c.params()[0].astype(np.float64), losses

    a, la = run(False)
    a2, la2 = run(False)
    b, lb = run(True)
    noise = np.abs(a2 - a)
    diff = np.abs(b - a)
    assert np.mean(diff) <= 3 * np.mean(noise) + 1e-9, (np.mean(diff), np.mean(noise))
    loss_noise = np.max(np.abs(la2 - la) / la)
    assert np.max(np.abs(lb - la) / la) <= 3 * loss_noise + 0.02, (la, la2, lb)
    assert la[-1] < la[0] and lb[-1] < lb[0]
