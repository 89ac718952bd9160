# -*- coding: utf-8 -*-
"""Kernels of the learned collision surrogate against the FP64 oracle
(GPU): windowed Hermite embedding and reconstruction, gate and device point
list,
the MLP's forward/backward/Adam kernels, and the assembled collide path.

Tolerances:
  embedding features/targets (FP32 outputs): 1e-5 normwise relative;
  frame moments (FP64): 1e-12;
  reconstruction: 1e-10 (FP64 banks), 2e-6 (FP32 banks);
  MLP gradients (BF16 weights, FP32 accumulation) against FP64 with the
  same BF16-rounded weights: 1e-4 normwise relative per tensor.
"""

import numpy as np
import pytest
import torch

from helpers import config, random_states, rel_err
from frfs_b200 import _lib
from frfs_b200.backend import B200Backend
from frfs_b200.scattering import DGFSVHSGLLScatteringModel
from frfs_b200.surrogate import MLP, VHSSurrogate, NFEAT, NMODES
from frfs_b200.velocitymesh import DGFSVelocityMesh
from oracle import surrogate as osur
from oracle import vhs as ovhs

pytestmark = pytest.mark.gpu


def _model(precision, name='couette-n24'):
    cfg = config(name, precision)
    be = B200Backend(cfg, device='cuda:0')
    vm = DGFSVelocityMesh(be, cfg)
    return be, vm, DGFSVHSGLLScatteringModel(be, cfg, vm)


def _bank(be, f):
    nupts, neles, V = f.shape
    return be.matrix((nupts, V, neles),
                     np.ascontiguousarray(f.transpose(0, 2, 1)))


def _near_eq(cv, n, seed, amp=0.02):
    """Maxwellians with random moments times a smooth small deviation."""
    rng = np.random.default_rng(seed)
    out = np.empty((n, cv.shape[1]))
    for i in range(n):
        rho, T = rng.uniform(0.6, 1.8), rng.uniform(0.7, 1.5)
        u = rng.uniform(-0.3, 0.3, 3)
        c = (cv - u[:, None])/np.sqrt(T)
        h = amp*(rng.standard_normal()*c[0]*c[1] +
                 rng.standard_normal()*c[2]*(np.sum(c*c, axis=0) - 2.5))
        out[i] = ovhs.maxwellian(cv, rho, u, T)*(1 + h)
    return out


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_embed_matches_oracle(precision):
    be, vm, sm = _model(precision)
    cv, cw = vm.cv(), vm.cw()
    nupts, neles = 2, 5
    f = random_states(cv, nupts*neles, seed=3).reshape(nupts, neles, -1)
    q = random_states(cv, nupts*neles, seed=4).reshape(nupts, neles, -1)
    fb, qb = _bank(be, f), _bank(be, q)
    sur = VHSSurrogate(sm)
    nub = sur.loss_rate(fb, be.matrix(fb.ioshape))
    X, B, mom, eps = sur.embed(fb, qb)
    _, Bg, _, _ = sur.embed(fb, qb, nubank=nub)
    torch.cuda.synchronize()
    X, B, Bg, mom, eps = (t.cpu().numpy() for t in (X, B, Bg, mom, eps))
    fu, qu = fb.get().astype(np.float64), qb.get().astype(np.float64)
    nu = nub.get().astype(np.float64)
    for u in range(nupts):
        for e in range(neles):
            pt = u*neles + e
            x, (rho, uu, T), ep, b = osur.embed(
                fu[u, :, e], cv, cw, vm.L(), Q=qu[u, :, e],
                prefac=sm.prefactor, gamma=sm._gamma)
            assert rel_err(mom[pt], np.r_[rho, uu, T]) < 1e-12
            assert rel_err(X[pt], x) < 1e-5
            assert rel_err(B[pt], b) < 1e-5
            assert abs(eps[pt] - ep) < 1e-5*ep
            _, _, _, bg = osur.embed(
                fu[u, :, e], cv, cw, vm.L(), Q=qu[u, :, e],
                prefac=sm.prefactor, gamma=sm._gamma, nu=nu[u, :, e])
            assert rel_err(Bg[pt], bg) < 1e-5


@pytest.mark.parametrize('precision', ['double', 'single'])
@pytest.mark.parametrize('name', ['relax0d-n16', 'couette-n24',
                                  'channel-n32'])
def test_loss_rate_matches_oracle(precision, name):
    """nu(c) = prefac Re IFFT(b2 FFT(f)/V), computed in FP32: 2e-6 of
    max nu; the gated call leaves the other points untouched."""
    be, vm, sm = _model(precision, name)
    from helpers import oracle_for
    ovm, pre, prefac = oracle_for(config(name, precision))
    nupts, neles = 1, 3
    f = random_states(vm.cv(), nupts*neles, seed=9).reshape(nupts, neles, -1)
    fb = _bank(be, f)
    sur = VHSSurrogate(sm)
    gate = torch.tensor([1, 0, 1], dtype=torch.int32, device=be.device)
    nub = sur.loss_rate(fb, be.matrix(fb.ioshape), gate)
    torch.cuda.synchronize()
    nu = nub.get()
    fu = fb.get().astype(np.float64)
    for e in range(neles):
        if e == 1:
            assert np.all(nu[0, :, e] == 0)
            continue
        _, lo = ovhs.vhs_Q_gain_loss(fu[0, :, e], ovm, pre, prefac)
        assert rel_err(nu[0, :, e], lo.real) < 2e-6


@pytest.mark.parametrize('precision', ['double', 'single'])
@pytest.mark.parametrize('coalesced', [False, True])
def test_reconstruct_matches_oracle_and_gate(precision, coalesced):
    """Per-point path for every gated point, or (coalesced) the split mode:
    the gate-1 points from a device list (in any order; the count caps it),
    the gate-2 points on the AoSoA kernels; 35 elements span two AoSoA
    blocks."""
    be, vm, sm = _model(precision)
    cv = vm.cv()
    nupts, neles = 1, 35
    npts = nupts*neles
    rng = np.random.default_rng(8)
    deg = np.array([sum(t) for t in osur.modes()])
    Bp = np.zeros((npts, NFEAT), np.float32)
    Bp[:, :NMODES] = rng.standard_normal((npts, NMODES))*0.5**deg
    mom = np.c_[rng.uniform(0.5, 2, npts), rng.uniform(-0.3, 0.3, (npts, 3)),
                rng.uniform(0.7, 1.5, npts)]
    gate = rng.choice([0, 1, 2, 2], npts).astype(np.int32)  # 2: loss term only
    gate[:3] = (0, 1, 2)
    dev = be.device
    out = be.matrix((nupts, vm.vsize(), neles))
    sur = VHSSurrogate(sm)
    d_b = torch.tensor(Bp, device=dev)
    d_mom = torch.tensor(mom, device=dev)
    d_gate = torch.tensor(gate, device=dev)
    Gw = osur.window_gram()
    d_gwinv = torch.tensor(np.linalg.inv(Gw).ravel(), device=dev)
    fh = random_states(cv, npts, seed=12).reshape(nupts, neles, -1)
    nh = np.abs(random_states(cv, npts, seed=13)).reshape(nupts, neles, -1)
    fb, nb = _bank(be, fh), _bank(be, 20*nh)
    work = torch.zeros(nupts*2*32*(32*5 + NMODES), dtype=torch.float64,
                       device=dev)
    net = np.nonzero(gate == 1)[0].astype(np.int32)
    d_net = torch.tensor(np.r_[net[::-1], -7], dtype=torch.int32, device=dev)
    d_nnet = torch.tensor([len(net)], dtype=torch.int32, device=dev)
    _lib.check(_lib.load().dgfs_hermite_reconstruct(
        be.precision, d_b.data_ptr(), d_mom.data_ptr(), d_gate.data_ptr(),
        nupts, neles, out.traits[1], vm.Nv(), vm.L(), vm.cw(), sm.prefactor,
        sm._gamma, sur.ginv.data_ptr(), d_gwinv.data_ptr(),
        fb._as_parameter_, nb._as_parameter_, out._as_parameter_,
        d_net.data_ptr() if coalesced else None,
        d_nnet.data_ptr() if coalesced else None,
        work.data_ptr() if coalesced else None, be.stream),
        'dgfs_hermite_reconstruct')
    torch.cuda.synchronize()
    Q = out.get()
    fu, nuu = fb.get().astype(np.float64), nb.get().astype(np.float64)
    tol = 1e-10 if precision == 'double' else 2e-6
    for pt in range(npts):
        u, e = divmod(pt, neles)
        if not gate[pt]:
            assert np.all(Q[u, :, e] == 0)
            continue
        b = Bp[pt].astype(np.float64)*(gate[pt] == 1)
        Qo = osur.reconstruct(b,
                              (mom[pt, 0], mom[pt, 1:4], mom[pt, 4]), cv,
                              sm.prefactor, sm._gamma, Gw=Gw, f=fu[u, :, e],
                              nu=nuu[u, :, e])
        assert rel_err(Q[u, :, e], Qo) < tol


def test_gate_builds_the_plain_list():
    dev = torch.device('cuda:0')
    rng = np.random.default_rng(2)
    eps = rng.uniform(0, 0.1, 1000).astype(np.float32)
    e = torch.tensor(eps, device=dev)
    gate = torch.empty(1000, dtype=torch.int32, device=dev)
    plain = torch.full((1000,), -1, dtype=torch.int32, device=dev)
    n = torch.empty(1, dtype=torch.int32, device=dev)
    net = torch.full((1000,), -1, dtype=torch.int32, device=dev)
    nn = torch.empty(1, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    mom = np.c_[np.ones(1000), rng.uniform(-1, 1, (1000, 3)),
                rng.uniform(0.5, 3, 1000)]
    d_mom = torch.tensor(mom, device=dev)
    L, rmin = 5.5, 3.5
    _lib.check(_lib.load().dgfs_surrogate_gate(
        1000, e.data_ptr(), 0.05, 0.01, d_mom.data_ptr(), L, rmin,
        gate.data_ptr(), plain.data_ptr(), n.data_ptr(), net.data_ptr(),
        nn.data_ptr(), s), 'dgfs_surrogate_gate')
    torch.cuda.synchronize()
    g = gate.cpu().numpy()
    res = (L - np.abs(mom[:, 1:4]).max(axis=1)) >= rmin*np.sqrt(mom[:, 4])
    assert 0 < res.sum() < 1000
    want = np.where(eps < np.float32(0.01), 2, 1)*(
        (eps < np.float32(0.05)) & res)
    assert np.array_equal(g, want.astype(np.int32))
    k = int(n.item())
    assert k == int(np.sum(g == 0))
    assert sorted(plain.cpu().numpy()[:k]) == list(np.nonzero(g == 0)[0])
    k = int(nn.item())
    assert k == int(np.sum(g == 1))
    assert sorted(net.cpu().numpy()[:k]) == list(np.nonzero(g == 1)[0])


def test_predict_on_a_row_list_matches_all_rows():
    """The network evaluated on a device row list (gather, GEMMs capped
    by a device count, scatter) gives the rows of the full evaluation bit
    for bit and leaves the other rows alone."""
    be, vm, sm = _model('single')
    sur = VHSSurrogate(sm, seed=3)
    dev = be.device
    g = torch.Generator(device='cpu').manual_seed(0)
    M = 300
    X = torch.randn(M, NFEAT, generator=g).to(dev)
    sur.mu_x = torch.randn(NFEAT, generator=g).to(dev)*0.1
    sur.is_x = (1 + torch.rand(NFEAT, generator=g)).to(dev)
    sur.mu_y = torch.randn(NFEAT, generator=g).to(dev)*0.1
    sur.is_y = (1 + torch.rand(NFEAT, generator=g)).to(dev)
    full = sur.predict(X).clone()
    rows = torch.tensor([5, 17, 299, 0, 123, 64, 65, 250], dtype=torch.int32,
                        device=dev)
    count = torch.tensor([6], dtype=torch.int32, device=dev)
    sur.ws.get('Bp', (M, NFEAT)).fill_(7.0)
    part = sur.predict(X, rows, count)
    torch.cuda.synchronize()
    used = rows[:6].long()
    assert torch.equal(part[used], full[used])
    rest = torch.ones(M, dtype=torch.bool, device=dev)
    rest[used] = False
    assert torch.all(part[rest] == 7.0)


@pytest.mark.parametrize('precision', ['double', 'single'])
def test_apply_list_matches_apply(precision):
    be, vm, sm = _model(precision, 'couette-n24' if precision == 'single'
                        else 'relax0d-n16')
    # 330 points: one whole-point launch for the bank (330 x 12 radial
    # chunks exceed the single-CTA kernel's split scratch), radial-node
    # chunks for the 17-point list; the two must agree bit for bit
    nupts, neles = 3, 110
    npts = nupts*neles
    f = random_states(vm.cv(), npts, seed=5).reshape(nupts, neles, -1)
    fin = _bank(be, f)
    full = be.matrix(fin.ioshape)
    sm.fs_all(fin, full)
    rng = np.random.default_rng(1)
    pts = rng.permutation(npts)[:17].astype(np.int32)
    pts_bad = np.r_[pts, npts + 5, -1].astype(np.int32)  # skipped entries
    dev = be.device
    d_pts = torch.tensor(pts_bad, device=dev)
    lib = _lib.load()
    ldim = fin.traits[1]
    out = be.matrix(fin.ioshape)
    _lib.check(lib.dgfs_vhs_apply_list(
        sm._h, fin._as_parameter_, out._as_parameter_, nupts, neles, ldim,
        be.soasz, d_pts.data_ptr(), None, len(pts_bad), be.stream),
        'dgfs_vhs_apply_list')
    # a device count caps the list at its first 5 entries
    cnt = torch.tensor([5], dtype=torch.int32, device=dev)
    out2 = be.matrix(fin.ioshape)
    _lib.check(lib.dgfs_vhs_apply_list(
        sm._h, fin._as_parameter_, out2._as_parameter_, nupts, neles, ldim,
        be.soasz, d_pts.data_ptr(), cnt.data_ptr(), len(pts), be.stream),
        'dgfs_vhs_apply_list')
    sm.status()
    Qf, Ql, Q5 = full.get(), out.get(), out2.get()
    for pt in range(npts):
        u, e = divmod(pt, neles)
        if pt in pts:
            assert np.array_equal(Ql[u, :, e], Qf[u, :, e])
        else:
            assert np.all(Ql[u, :, e] == 0)
        if pt in pts[:5]:
            assert np.array_equal(Q5[u, :, e], Qf[u, :, e])
        else:
            assert np.all(Q5[u, :, e] == 0)
    with pytest.raises(_lib.DgfsError):
        _lib.check(lib.dgfs_vhs_apply_list(
            sm._h, fin._as_parameter_, out._as_parameter_, nupts, neles,
            ldim, be.soasz, None, None, 3, be.stream), 'dgfs_vhs_apply_list')


def _bf16(t):
    return t.to(torch.bfloat16).to(torch.float64).cpu().numpy()


@pytest.mark.parametrize('tc', [False, 'staged', 'tma'])
def test_mlp_gradients_match_oracle(tc):
    """SIMT products (FP32 activations) against the FP64 oracle with the
    same BF16 weights at 1e-4.  Tensor-core products (BF16 operands)
    against the oracle that rounds the same operands at 4e-3: the GPU's
    FP32 activations and the oracle's FP64 ones can round to neighbouring
    BF16 values, one BF16 step (2^-8) in a few operands; and against the
    unrounded oracle at 1.5e-2, the size of BF16 operand rounding."""
    dev = torch.device('cuda:0')
    mlp = MLP(dev, seed=4, tc=tc)
    rng = np.random.default_rng(6)
    for k in ('b1', 'b2', 'b3', 'b4'):
        mlp.w[k].copy_(torch.tensor(0.1*rng.standard_normal(mlp.w[k].shape)))
    mlp.w['Ws'].copy_(torch.tensor(
        0.05*rng.standard_normal(mlp.w['Ws'].shape)))
    mlp.sync_bf16()
    Bt = 70                                   # not a multiple of the tile
    X = torch.tensor(rng.standard_normal((Bt, NFEAT)), dtype=torch.float32,
                     device=dev)
    T = torch.tensor(rng.standard_normal((Bt, NFEAT)), dtype=torch.float32,
                     device=dev)
    w = torch.tensor(rng.uniform(0.5, 2, NFEAT), dtype=torch.float32,
                     device=dev)
    Y = mlp.forward(X, keep=True)
    dY = torch.empty_like(Y)
    rl = torch.empty(Bt, dtype=torch.float64, device=dev)
    _lib.check(_lib.load().dgfs_mlp_mse(
        Bt, NFEAT, NMODES, Y.data_ptr(), T.data_ptr(), w.data_ptr(),
        dY.data_ptr(), rl.data_ptr(), torch.cuda.current_stream().cuda_stream),
        'dgfs_mlp_mse')
    g = mlp.backward(dY)
    torch.cuda.synchronize()
    P = [(_bf16(mlp.w[k]) if k.startswith('W') else
          mlp.w[k].double().cpu().numpy()) for k in MLP.names]
    Xn = X.double().cpu().numpy()
    rnd = osur.bf16_round if tc else None
    tol = 4e-3 if tc else 1e-4
    Yo, cache = osur.mlp_forward(P, Xn, rnd=rnd)
    loss, dYo = osur.mse(Yo, T.double().cpu().numpy(), NMODES,
                         w.double().cpu().numpy())
    assert rel_err(Y.cpu().numpy(), Yo) < tol
    assert abs(float(rl.sum())/(Bt*NMODES) - loss) < tol*loss
    go = osur.mlp_backward(P, cache, dYo, rnd=rnd)
    for k in MLP.names:
        assert rel_err(g[k].cpu().numpy(), go[k]) < tol, k
    if tc:
        Yu, cu = osur.mlp_forward(P, Xn)
        gu = osur.mlp_backward(P, cu, osur.mse(
            Yu, T.double().cpu().numpy(), NMODES,
            w.double().cpu().numpy())[1])
        assert rel_err(Y.cpu().numpy(), Yu) < 1.5e-2
        for k in MLP.names:
            assert rel_err(g[k].cpu().numpy(), gu[k]) < 1.5e-2, k
        mlp.check_tc()


def test_scheduled_adam_matches_per_tensor_adam():
    """One Adam launch over the flat buffer at the device schedule's rate
    equals the per-tensor launches at the host-computed rate (weight decay
    on the weights only); the schedule's counters advance."""
    dev = torch.device('cuda:0')
    a, b = MLP(dev, seed=2), MLP(dev, seed=2)
    rng = np.random.default_rng(3)
    lr, lr_min, total, wd = 2e-3, 0.1, 7, 1e-3
    b.start_schedule()
    for it in range(3):
        for k in MLP.names:
            gk = torch.tensor(rng.standard_normal(a.g[k].shape),
                              dtype=torch.float32)
            a.g[k].copy_(gk)
            b.g[k].copy_(gk)
        frac = it/total
        a.adam(lr=lr*(lr_min + (1 - lr_min)*0.5*(1 + np.cos(np.pi*frac))),
               wd=wd)
        b.adam_scheduled(lr, lr_min, total, wd=wd)
    torch.cuda.synchronize()
    for k in MLP.names:
        assert rel_err(b.w[k].cpu().numpy(), a.w[k].cpu().numpy()) < 1e-6, k
        if k.startswith('W'):
            assert torch.equal(b.wb[k], b.w[k].to(torch.bfloat16)), k
    assert b.counters.cpu().tolist() == [3, 3]


def test_graph_training_equals_eager_training():
    """The CUDA-graph replay of the training step gives bit-identical
    weights and losses to running every step eagerly."""
    dev = torch.device('cuda:0')
    be, vm, sm = _model('single')
    rng = np.random.default_rng(8)
    n = 2048
    X = torch.tensor(rng.standard_normal((n, NFEAT)), dtype=torch.float32,
                     device=dev)
    Y = torch.tensor(rng.standard_normal((n, NFEAT)), dtype=torch.float32,
                     device=dev)
    out = []
    for graph in (False, True):
        sur = VHSSurrogate(sm, seed=5)
        sur.set_normalisation(X, Y)
        hist = sur.train(X, Y, epochs=3, batch=256, lr=1e-3, graph=graph)
        out.append((hist, sur.mlp.state(), sur.mlp.step))
    assert out[0][0] == out[1][0]
    assert out[0][2] == out[1][2] == 3*(n//256)
    for k in MLP.names:
        assert np.array_equal(out[0][1][k], out[1][1][k]), k


def test_adam_step_matches_formula():
    dev = torch.device('cuda:0')
    rng = np.random.default_rng(9)
    n = 1000
    w0, g0 = rng.standard_normal(n), rng.standard_normal(n)
    w = torch.tensor(w0, dtype=torch.float32, device=dev)
    wb = torch.empty(n, dtype=torch.bfloat16, device=dev)
    g = torch.tensor(g0, dtype=torch.float32, device=dev)
    m1, m2 = torch.zeros_like(w), torch.zeros_like(w)
    s = torch.cuda.current_stream().cuda_stream
    lib = _lib.load()
    mo1, mo2 = np.zeros(n), np.zeros(n)
    wo = w0.astype(np.float32).astype(np.float64)
    for step in (1, 2, 3):
        _lib.check(lib.dgfs_mlp_adam(n, w.data_ptr(), wb.data_ptr(),
                                     g.data_ptr(), m1.data_ptr(),
                                     m2.data_ptr(), 1e-2, 0.9, 0.999, 1e-8,
                                     step, 1e-3, s), 'dgfs_mlp_adam')
        gi = g0.astype(np.float32) + 1e-3*wo
        mo1 = 0.9*mo1 + 0.1*gi
        mo2 = 0.999*mo2 + 0.001*gi*gi
        wo = wo - 1e-2*(mo1/(1 - 0.9**step))/(np.sqrt(mo2/(1 - 0.999**step))
                                              + 1e-8)
    torch.cuda.synchronize()
    assert np.max(np.abs(w.cpu().numpy() - wo)) < 1e-5
    assert torch.equal(wb, w.to(torch.bfloat16))


def test_training_reduces_loss():
    """A learnable synthetic map (linear part plus a tanh part) is fitted
    by the project's kernels: the loss falls by more than 10x."""
    dev = torch.device('cuda:0')
    be, vm, sm = _model('single')
    sur = VHSSurrogate(sm, seed=1)
    rng = np.random.default_rng(0)
    n = 8192
    Xh = rng.standard_normal((n, NFEAT))
    A = rng.standard_normal((NFEAT, NFEAT))/np.sqrt(NFEAT)
    C = rng.standard_normal((NFEAT, NFEAT))/np.sqrt(NFEAT)
    Yh = Xh @ A + 0.3*np.tanh(Xh @ C)
    X = torch.tensor(Xh, dtype=torch.float32, device=dev)
    Y = torch.tensor(Yh, dtype=torch.float32, device=dev)
    sur.set_normalisation(X, Y)
    hist = sur.train(X, Y, epochs=20, batch=512, lr=2e-3)
    assert hist[-1] < 0.1*hist[0], hist


def test_collide_routes_points_and_conserves():
    """threshold 0: every point takes the plain operator (bit-identical to
    fs_all); threshold huge: every resolved point takes the network and its
    Q has zero mass, momentum and energy; in between the routing follows
    eps."""
    be, vm, sm = _model('single')
    cv = vm.cv()
    nupts, neles = 3, 12
    npts = nupts*neles
    f = np.concatenate([_near_eq(cv, npts - 8, seed=2),
                        random_states(cv, 8, seed=3)]).reshape(
                            nupts, neles, -1)
    fb = _bank(be, f)
    sur = VHSSurrogate(sm, seed=0)
    # the plain points must equal the fallback handle's own evaluation
    ref = be.matrix(fb.ioshape)
    _lib.check(_lib.load().dgfs_vhs_apply(
        sur._plain_h, fb._as_parameter_, ref._as_parameter_, nupts, neles,
        fb.traits[1], be.soasz, -1, 0, be.stream), 'dgfs_vhs_apply')
    out = be.matrix(fb.ioshape)
    g = sur.collide(fb, out, threshold=0.0)
    torch.cuda.synchronize()
    assert int(g.sum()) == 0
    assert np.array_equal(out.get(), ref.get())

    _, _, mom, eps = sur.embed(fb)
    e = eps.cpu().numpy()
    res = sur.resolved(mom).cpu().numpy()
    assert res.sum() >= npts - 4
    out2 = be.matrix(fb.ioshape)
    g = (sur.collide(fb, out2, threshold=1e30).cpu().numpy() != 0)
    torch.cuda.synchronize()
    assert np.array_equal(g, res)
    Q = out2.get().astype(np.float64)
    phi = np.vstack([np.ones(cv.shape[1]), cv, np.sum(cv*cv, axis=0)])
    for u in range(nupts):
        for el in range(neles):
            if not g[u*neles + el]:
                continue
            m = phi @ Q[u, :, el]
            scale = np.abs(phi) @ np.abs(Q[u, :, el])
            assert np.all(np.abs(m) < 1e-5*scale)

    thr = float(np.median(e))
    out3 = be.matrix(fb.ioshape)
    g = (sur.collide(fb, out3, threshold=thr).cpu().numpy() != 0)
    torch.cuda.synchronize()
    assert np.array_equal(g, (e < np.float32(thr)) & res)
    Q3, Qr, Q2 = out3.get(), ref.get(), out2.get()
    for pt in range(npts):
        u, el = divmod(pt, neles)
        want = Q2 if g[pt] else Qr
        assert np.array_equal(Q3[u, :, el], want[u, :, el])
    assert sur.residual_check(fb, out3, be.matrix(fb.ioshape)) > 0


def test_scale_rows_matches_numpy():
    """Scale-free rows: degree >= 2 columns divided by max(eps, 1e-3), log
    of that scale in the spare column; the inverse multiplies back."""
    dev = torch.device('cuda:0')
    rng = np.random.default_rng(4)
    M = 300
    X = rng.standard_normal((M, NFEAT)).astype(np.float32)
    eps = np.abs(rng.standard_normal(M)).astype(np.float32)*0.05
    eps[:10] = 1e-5                                   # below the floor
    d_x = torch.tensor(X, device=dev)
    d_e = torch.tensor(eps, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    lib = _lib.load()
    _lib.check(lib.dgfs_surrogate_scale(M, NFEAT, d_e.data_ptr(), 1e-3, 4,
                                        NMODES, 224, 0, d_x.data_ptr(), s),
               'dgfs_surrogate_scale')
    sc = np.maximum(eps, np.float32(1e-3))
    want = X.copy()
    want[:, 4:NMODES] /= sc[:, None]
    want[:, 224] = np.log(sc)
    got = d_x.cpu().numpy()
    assert np.allclose(got, want, rtol=1e-6, atol=1e-7)
    _lib.check(lib.dgfs_surrogate_scale(M, NFEAT, d_e.data_ptr(), 1e-3, 0,
                                        NMODES, -1, 1, d_x.data_ptr(), s),
               'dgfs_surrogate_scale')
    want[:, :NMODES] *= sc[:, None]
    assert np.allclose(d_x.cpu().numpy(), want, rtol=1e-6, atol=1e-7)
    with pytest.raises(_lib.DgfsError):   # log column inside the range
        _lib.check(lib.dgfs_surrogate_scale(M, NFEAT, d_e.data_ptr(), 1e-3,
                                            0, NMODES, 10, 0, d_x.data_ptr(),
                                            s), 'dgfs_surrogate_scale')
