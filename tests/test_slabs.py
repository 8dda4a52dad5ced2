"""z-slab decomposition of one grid (gdiamond_b200/slabs.py) on the CPU.

* HaloPlan: owned ranges partition the grid, local ranges add `halo` planes on inner sides,
  every send has the matching receive;
* the decomposition run with the oracle as each part's stepper -- blocks of `halo` steps, halo
  exchange after each -- reproduces the single-grid oracle bit for bit (fields and a DFT
  monitor), with a point source inside a neighbour's halo and a plane source; a halo one
  plane short on the upper side does not;
* the same exchange between processes over torch.distributed (gloo, 2 and 3 ranks) through
  exchange_dist, the function the multi-GPU run uses over NCCL.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from gdiamond_b200 import slabs as Z
from gdiamond_b200 import workloads as W

SHAPE = (14, 12, 23)
T = 9


def test_plan_partition_and_symmetry():
    for nz, parts, halo in [(23, 3, 2), (64, 4, 3), (10, 2, 1), (9, 1, 2), (12, 3, 3)]:
        p = Z.HaloPlan(nz, parts, halo)
        assert p.own[0][0] == 0 and p.own[-1][1] == nz
        for r in range(parts - 1):
            assert p.own[r][1] == p.own[r + 1][0]
        for r in range(parts):
            lo, hi = p.own[r]
            assert hi - lo >= halo + 1
            assert p.loc[r] == (lo - halo if r else 0, hi + halo + 1 if r < parts - 1 else nz)
            for peer, k0, nk in p.sends(r):
                assert (r, k0, nk) in p.recvs(peer)
                assert p.own[r][0] <= k0 and k0 + nk <= p.own[r][1]      # sends owned planes
                assert p.to_local(peer, k0) is not None                  # into the peer's halo
                assert not (p.own[peer][0] <= k0 < p.own[peer][1])
    with pytest.raises(ValueError):
        Z.HaloPlan(5, 3, 2)


def problem():
    eps = W.spheres_eps(SHAPE, n_spheres=4, r_range=(2, 4), seed=7)
    coefs = W.reference_coefficients(SHAPE, eps_re=eps, t_pml=3)
    w = W.gaussian_wave(T, delay=4.0, width=2.0, period=5.0)
    nx, ny, nz = SHAPE
    sources = [dict(component="Jz", wave=w, i=nx // 2, j=ny // 2, k=8),   # in part 1's halo
               dict(component="Mx", wave=w * np.float32(0.5), i=3, j=4, k=15),
               dict(component="Jx", wave=w * np.float32(0.1), k=5, kind=1)]
    freqs = W.source_band(3, period=5.0, width=2.0)
    return coefs, sources, freqs


def osrc(s):
    return oracle.Source(s["component"], s["wave"], i=s.get("i", 0), j=s.get("j", 0), k=s["k"],
                         kind=s.get("kind", 0))


def single_grid(coefs, sources, freqs, mon_k):
    mon = oracle.Monitor("Ez", mon_k, freqs, 1.0)
    F = oracle.run(SHAPE, coefs, T, sources=[osrc(s) for s in sources], monitors=[mon])
    return F, mon


class OraclePart:
    """One part of the decomposition stepped by the oracle."""

    def __init__(self, plan, r, coefs, sources, freqs, mon_k):
        nx, ny, _ = SHAPE
        self.plan, self.r = plan, r
        lo, hi = plan.loc[r]
        self.lo, self.shape = lo, (nx, ny, hi - lo)
        self.coefs = [Z.slice_planes(c, SHAPE, lo, hi) for c in coefs]
        self.sources = [osrc(s) for s in Z.localize_sources(plan, r, sources)]
        self.mon = None
        if plan.owner(mon_k) == r:
            self.mon = oracle.Monitor("Ez", plan.to_local(r, mon_k), freqs, 1.0)
        self.F = [np.zeros(nx * ny * (hi - lo), np.float32) for _ in range(6)]
        self.t = 0

    def step(self, b):
        self.F = oracle.run(self.shape, self.coefs, b, sources=self.sources,
                            monitors=[self.mon] if self.mon else [], fields=self.F, t0=self.t)
        self.t += b

    def planes(self, k0, nk):
        nx, ny, nz = self.shape
        return np.stack([f.reshape(nz, ny, nx)[k0 - self.lo:k0 - self.lo + nk] for f in self.F])

    def put(self, k0, nk, block):
        nx, ny, nz = self.shape
        for c in range(6):
            self.F[c].reshape(nz, ny, nx)[k0 - self.lo:k0 - self.lo + nk] = block[c]

    def owned(self):
        nx, ny, nz = self.shape
        lo, hi = self.plan.own[self.r]
        return [f.reshape(nz, ny, nx)[lo - self.lo:hi - self.lo] for f in self.F]


def check_against_single(parts_owned, mon_parts, plan, coefs, sources, freqs, mon_k):
    F_ref, mon_ref = single_grid(coefs, sources, freqs, mon_k)
    nx, ny, nz = SHAPE
    for c in range(6):
        got = np.concatenate([o[c] for o in parts_owned]).reshape(-1)
        assert np.array_equal(got.view(np.uint32), F_ref[c].view(np.uint32)), oracle.COMPONENTS[c]
    re, im = mon_parts
    assert np.abs(mon_ref.re).max() > 0
    assert np.array_equal(re, mon_ref.re) and np.array_equal(im, mon_ref.im)


@pytest.mark.parametrize("parts,halo", [(3, 2), (2, 3), (4, 1), (5, 3)])
def test_decomposition_matches_single_grid(parts, halo):
    coefs, sources, freqs = problem()
    mon_k = 12
    plan = Z.HaloPlan(SHAPE[2], parts, halo)
    P = [OraclePart(plan, r, coefs, sources, freqs, mon_k) for r in range(parts)]
    done = 0
    while done < T:  # T = 9: a short last block when halo does not divide it
        b = min(halo, T - done)
        for p in P:
            p.step(b)
        for p in P:
            for peer, k0, nk in plan.sends(p.r):
                P[peer].put(k0, nk, p.planes(k0, nk))
        done += b
    owner = P[plan.owner(mon_k)].mon
    check_against_single([p.owned() for p in P], (owner.re, owner.im), plan, coefs, sources,
                         freqs, mon_k)


class SymmetricPlan(Z.HaloPlan):
    """The same split with `halo` planes on both sides: one plane short above."""

    def __init__(self, nz, parts, halo):
        super().__init__(nz, parts, halo)
        self.loc = [(lo, hi - 1 if r < parts - 1 else hi) for r, (lo, hi) in enumerate(self.loc)]

    def sends(self, r):
        return [(p, k0 if p > r else k0, self.halo) for p, k0, _ in super().sends(r)]

    def recvs(self, r):
        return [(p, k0, self.halo) for p, k0, _ in super().recvs(r)]


def run_parts(plan, coefs, sources, freqs, mon_k):
    P = [OraclePart(plan, r, coefs, sources, freqs, mon_k) for r in range(plan.parts)]
    done = 0
    while done < T:
        b = min(plan.halo, T - done)
        for p in P:
            p.step(b)
        for p in P:
            for peer, k0, nk in plan.sends(p.r):
                P[peer].put(k0, nk, p.planes(k0, nk))
        done += b
    return [p.owned() for p in P]


def test_upper_halo_needs_one_more_plane():
    coefs, sources, freqs = problem()
    F_ref, _ = single_grid(coefs, sources, freqs, 12)
    plan = SymmetricPlan(SHAPE[2], 3, 2)
    owned = run_parts(plan, coefs, sources, freqs, 12)
    bad = [c for c in range(6)
           if not np.array_equal(np.concatenate([o[c] for o in owned]).reshape(-1), F_ref[c])]
    assert bad, "a symmetric halo should corrupt the planes below each upper slab boundary"


def _worker(rank, world, port, halo, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    coefs, sources, freqs = problem()
    mon_k = 12
    plan = Z.HaloPlan(SHAPE[2], world, halo)
    part = OraclePart(plan, rank, coefs, sources, freqs, mon_k)
    nx, ny, _ = SHAPE
    done = 0
    while done < T:
        b = min(halo, T - done)
        part.step(b)
        Z.exchange_dist(plan, rank,
                        lambda k0, nk: torch.from_numpy(part.planes(k0, nk).view(np.int32)),
                        lambda k0, nk, buf: part.put(k0, nk, buf.numpy().view(np.float32)),
                        lambda nk: torch.empty((6, nk, ny, nx), dtype=torch.int32))
        done += b
    np.savez(os.path.join(outdir, f"part{rank}.npz"), *part.owned(),
             re=part.mon.re if part.mon else np.zeros(0), im=part.mon.im if part.mon else np.zeros(0))
    dist.barrier()
    dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("world,halo", [(2, 2), (3, 3)])
def test_exchange_over_gloo_matches_single_grid(tmp_path, world, halo):
    mp.spawn(_worker, args=(world, free_port(), halo, str(tmp_path)), nprocs=world, join=True)
    coefs, sources, freqs = problem()
    mon_k = 12
    plan = Z.HaloPlan(SHAPE[2], world, halo)
    owned, mon = [], None
    for r in range(world):
        d = np.load(tmp_path / f"part{r}.npz")
        owned.append([d[f"arr_{c}"] for c in range(6)])
        if plan.owner(mon_k) == r:
            mon = (d["re"], d["im"])
    check_against_single(owned, mon, plan, coefs, sources, freqs, mon_k)
