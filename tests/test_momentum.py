"""Channel momentum ADI sweeps (btdma_momentum_*) against the CPU restatement of
the reference's build + TDMA + scatter, per direction and component, and the
full z -> y -> x step; periodic x / y, stretched no-slip z.  Bar: 1e-12
relative (PaScaL sweeps vs the oracle's serial Thomas)."""
import numpy as np
import pytest

from oracle import momentum_oracle as MO


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.gpu
@pytest.mark.parametrize("direction", [0, 1, 2])
@pytest.mark.parametrize("comp", [0, 1, 2])
def test_sweep_matches_oracle(cuda, orc, direction, comp):
    import torch
    from filtered_tdma_b200.momentum import ChannelMomentum
    m = ChannelMomentum(64, 32, 48, gamma3=1.5)
    rng = np.random.default_rng(10 + 3 * direction + comp)
    q = rng.uniform(-1, 1, m.shape)
    c = 0.5 * (1.0 / 180.0) * 2e-3 * 50  # nu dt / 2, strong enough to matter
    dq = torch.from_numpy(q).to(cuda)
    out = torch.from_numpy(q).to(cuda)
    m.sweep(direction, comp, dq, out, c)
    torch.cuda.synchronize()
    assert m.status() == 0
    ref = MO.sweep(q, m.metrics, direction, comp, c, direction < 2)
    got = out.cpu().numpy()
    assert _rel(got[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1]) <= 1e-12
    assert np.array_equal(got[0], q[0])  # ghosts untouched


@pytest.mark.gpu
@pytest.mark.parametrize("comp", [0, 2])
def test_adi_benched_256_axes_matches_oracle(cuda, orc, comp):
    # the benched channel grid's sweep length, 256 rows (16 sub-segments) along
    # every axis: periodic x and y, stretched walls in z; the z sweep's systems
    # span the full 256 x 256 plane, x and y are thinner to keep the oracle short
    import torch
    from filtered_tdma_b200.momentum import ChannelMomentum
    c = 0.5 * (1.0 / 180.0) * 1e-3 * 50
    for nx, ny, nz in ((256, 256, 32), (32, 256, 256), (256, 32, 256)):
        m = ChannelMomentum(nx, ny, nz, gamma3=1.5)
        rng = np.random.default_rng(50 + nx + 2 * ny + 3 * nz + comp)
        rhs = rng.uniform(-1, 1, m.shape)
        d_rhs = torch.from_numpy(rhs).to(cuda)
        d_q = torch.zeros_like(d_rhs)
        m.adi(comp, d_rhs, d_q, c)
        torch.cuda.synchronize()
        assert m.status() == 0
        ref = MO.adi(rhs, m.metrics, comp, c, (True, True))
        assert _rel(d_q.cpu().numpy()[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1]) <= 1e-12
        m.close()


@pytest.mark.gpu
def test_adi_matches_oracle_walls_only(cuda, orc):
    import torch
    from filtered_tdma_b200.momentum import ChannelMomentum
    m = ChannelMomentum(32, 48, 64, gamma3=2.0, pbc_x=False, pbc_y=False)
    rng = np.random.default_rng(21)
    rhs = rng.uniform(-1, 1, m.shape)
    c = 0.05
    for comp in (0, 2):
        d_rhs = torch.from_numpy(rhs).to(cuda)
        d_q = torch.zeros_like(d_rhs)
        m.adi(comp, d_rhs, d_q, c)
        torch.cuda.synchronize()
        ref = MO.adi(rhs, m.metrics, comp, c, (False, False))
        assert _rel(d_q.cpu().numpy()[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1]) <= 1e-12


@pytest.mark.gpu
def test_factor_tables_follow_the_coefficient(cuda, orc):
    # one handle, the coefficient changing between calls, repeated, and a call
    # on another stream: each (dir, comp) factor table is reused only for the
    # coefficient and stream it was built for
    import torch
    from filtered_tdma_b200.momentum import ChannelMomentum
    m = ChannelMomentum(64, 32, 48, gamma3=1.5)
    rng = np.random.default_rng(33)
    q = rng.uniform(-1, 1, m.shape)
    side = torch.cuda.Stream()
    for c, stream in ((0.05, None), (0.2, None), (0.05, None), (0.05, None), (0.2, side)):
        for direction in (0, 1, 2):
            dq = torch.from_numpy(q).to(cuda)
            out = torch.from_numpy(q).to(cuda)
            torch.cuda.synchronize()
            m.sweep(direction, 1, dq, out, c, stream=0 if stream is None else stream.cuda_stream)
            torch.cuda.synchronize()
            ref = MO.sweep(q, m.metrics, direction, 1, c, direction < 2)
            assert _rel(out.cpu().numpy()[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1]) <= 1e-12
    assert m.status() == 0


@pytest.mark.gpu
def test_graph_replays_leave_the_cached_tables_alone(cuda, orc):
    # normal call with c1 (caches its tables), capture with c2, normal call with
    # c1, replay the c2 graph, normal call with c1 again: the last call must
    # still use c1's tables (bit-identical to a fresh handle), and the replay
    # must give c2's solution
    import torch
    from filtered_tdma_b200.momentum import ChannelMomentum
    m = ChannelMomentum(64, 32, 48, gamma3=1.5)
    fresh = ChannelMomentum(64, 32, 48, gamma3=1.5)
    rng = np.random.default_rng(44)
    q = rng.uniform(-1, 1, m.shape)
    c1, c2 = 0.05, 0.2
    stream = torch.cuda.Stream()
    s = stream.cuda_stream
    for direction in (2, 1, 0):
        dq = torch.from_numpy(q).to(cuda)
        out = torch.zeros_like(dq)
        gout = torch.zeros_like(dq)
        with torch.cuda.stream(stream):
            m.sweep(direction, 1, dq, out, c1, stream=s)
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            m.sweep(direction, 1, dq, gout, c2, stream=s)
        with torch.cuda.stream(stream):
            m.sweep(direction, 1, dq, out, c1, stream=s)
            g.replay()
            m.sweep(direction, 1, dq, out, c1, stream=s)
        stream.synchronize()
        want = torch.zeros_like(dq)
        fresh.sweep(direction, 1, dq, want, c1)
        torch.cuda.synchronize()
        assert torch.equal(out, want)
        ref2 = MO.sweep(q, m.metrics, direction, 1, c2, direction < 2)
        assert _rel(gout.cpu().numpy()[1:-1, 1:-1, 1:-1], ref2[1:-1, 1:-1, 1:-1]) <= 1e-12
        del g
    assert m.status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("direction", [0, 1, 2])
def test_filtered_backend_one_segment_is_serial_thomas(cuda, orc, direction):
    # the reference's channel on one rank: FilteredTDMACUDA with nprocs = 1
    # falls back to the serial Thomas; P = 1 here is bit-identical to it
    import torch
    from filtered_tdma_b200.momentum import ChannelMomentum
    m = ChannelMomentum(64, 32, 48, gamma3=1.5)
    m.set_backend("filtered", P=1, eps_constant=1e-3)
    rng = np.random.default_rng(70 + direction)
    q = rng.uniform(-1, 1, m.shape)
    c = 0.5 * (1.0 / 180.0) * 2e-3 * 50
    for comp in (0, 2):
        dq = torch.from_numpy(q).to(cuda)
        out = torch.from_numpy(q).to(cuda)
        m.sweep(direction, comp, dq, out, c)
        torch.cuda.synchronize()
        ref = MO.sweep(q, m.metrics, direction, comp, c, direction < 2)
        assert np.array_equal(out.cpu().numpy(), ref)
    assert m.status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("direction", [0, 1, 2])
def test_filtered_backend_segments(cuda, orc, direction):
    # Filtered v2 over 4 segments: with the reference-order flag bit-identical
    # to the oracle's Filtered v2 on the same A, B, C, D (rho from system 0's
    # column, the device J estimator, eps_constant as given); by default, where
    # every segment truncates, the tiled kernels' Filtered (exact segments, 2x2
    # interfaces: within eps of the serial Thomas solution), the exact solve
    # where one does not
    import torch
    from filtered_tdma_b200 import _lib as L
    from filtered_tdma_b200.momentum import ChannelMomentum
    rng = np.random.default_rng(80 + direction)
    for c, eps_c in ((0.5 * (1.0 / 180.0) * 2e-3 * 50, 1e-3), (0.5, 1e-3)):
        for flags in (L.FLAG_REFERENCE_ORDER, 0):
            m = ChannelMomentum(64, 64, 64, gamma3=1.5)
            m.set_backend("filtered_v2", P=4, flags=flags, eps_constant=eps_c)
            q = rng.uniform(-1, 1, m.shape)
            dq = torch.from_numpy(q).to(cuda)
            out = torch.from_numpy(q).to(cuda)
            m.sweep(direction, 1, dq, out, c)
            torch.cuda.synchronize()
            assert m.status() == 0
            got = out.cpu().numpy()
            Js = []

            def filt(A, B, C, D, periodic):
                x, J = orc.filtered(A, B, C, D, 4, 2, periodic, eps_c,
                                    orc.rho_rows(A, B, C, 0), orc.J_DEVICE)
                Js.append(list(J))
                return x

            ref = MO.sweep(q, m.metrics, direction, 1, c, direction < 2, solver=filt)
            exact = flags == 0 and max(Js[0]) >= 64 // 4 - 2
            if flags == 0:
                xt = MO.sweep(q, m.metrics, direction, 1, c, direction < 2)
                if exact:
                    assert _rel(got[1:-1, 1:-1, 1:-1], xt[1:-1, 1:-1, 1:-1]) <= 1e-12
                else:
                    eps = eps_c / 64.0 ** 2
                    assert np.max(np.abs(got - xt)) <= eps
                    assert np.max(np.abs(got - ref)) <= 2 * eps
            else:
                assert np.array_equal(got, ref)
            m.close()


def test_momentum_argument_checks():
    import ctypes
    from filtered_tdma_b200 import _lib as L
    z = np.zeros(100)
    h = ctypes.c_void_p()
    p = z.ctypes.data
    assert L.lib().btdma_momentum_create(30, 32, 32, p, p, p, p, p, p, 1, 1,
                                         ctypes.byref(h)) == L.ERR_UNSUPPORTED
    assert L.lib().btdma_momentum_create(48, 32, 32, p, p, p, p, p, p, 1, 1,
                                         ctypes.byref(h)) == L.ERR_UNSUPPORTED  # 48/16 not 2^k
    assert L.lib().btdma_momentum_sweep(None, 0, 0, None, None, 0.1, None) == L.ERR_ARG
    assert L.lib().btdma_momentum_set_backend(None, 2, 4, 0, 1e-3) == L.ERR_ARG


@pytest.mark.gpu
def test_adi_bit_identical_over_repeats_and_handles(cuda):
    # z -> y -> x at 256^3 (the benched grid): the sweeps' groups share shared
    # memory and warps run ahead of one another, so a race between them would
    # show as runs that differ.  Repeats on one handle and fresh handles must
    # agree bit for bit, for the staged-store sweeps (x, y) and the field-box
    # z sweep.
    import torch
    from filtered_tdma_b200.momentum import ChannelMomentum
    c = 0.5 * (1.0 / 180.0) * 1e-3 * 50
    g = torch.Generator(device=cuda)
    g.manual_seed(11)
    first = ChannelMomentum(256, 256, 256, gamma3=1.5)
    rhs = torch.rand(first.shape, dtype=torch.float64, device=cuda, generator=g)
    outs = []
    for handle in range(3):
        m = first if handle == 0 else ChannelMomentum(256, 256, 256, gamma3=1.5)
        for _ in range(3 if handle == 0 else 1):
            q = torch.zeros_like(rhs)
            m.adi(0, rhs, q, c)
            torch.cuda.synchronize()
            assert m.status() == 0
            outs.append(q)
        m.close()
    assert all(torch.equal(o, outs[0]) for o in outs[1:])
