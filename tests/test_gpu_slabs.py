"""j slabs on one GPU: the tiles of a domain, each a context with stored j ghost
planes, stepped in one process with the halo exchange between their buffers
(lbm_b200.slabs.step_local).  Checked against the same tiling composed from the
oracle's routines (postcoll, solids, boundarycond per tile, the exchange of
m_mpi_halo_exchange_j.F90, then drift and macrovars), FP32 and FP64, with the
floor rule of the fused tests.  The reference's tiles apply their own periodic
j copies before the exchange, so with closed k faces a tiled run differs from
the undivided domain next to the tile seams; with periodic k it does not, and
there the tiles must reproduce the undivided GPU run bit for bit."""
import numpy as np
import pytest

from lbm_b200 import workloads as W
from oracle import oracle as O
from tests.test_gpu_fused import compare_to_floor, cuda, host, params_of

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def global_start(wl):
    """An initialised global state (reference init order) in FP64, the blanking and uvel."""
    cfg = O.Config(wl.nx, wl.ny, wl.nz, wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=3,
                   lsolids=True, kinevisc=wl.kinevisc, smagorinsky=wl.smagorinsky)
    o = O.Oracle(cfg, np.float64)
    rho, u, v, w = (a.astype(np.float64) for a in W.initial_macro(wl))
    uvel = W.inflow_profile(wl, np.float64)
    fA, fB = o.zeros_f(), o.zeros_f()
    o.init(fA, fB, rho, u, v, w, uvel)
    R = [o.zeros_s() for _ in range(4)]
    o.macrovars(*R, fA)
    return fA, fB, R, W.blanking(wl), uvel


def oracle_tiles(wl, ntiles, dtype, steps):
    from lbm_b200 import slabs
    fA, fB, R, blank, uvel = global_start(wl)
    ny = wl.ny // ntiles
    cfg = O.Config(wl.nx, ny, wl.nz, wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=3, lsolids=True,
                   kinevisc=wl.kinevisc, smagorinsky=wl.smagorinsky)
    tiles = []
    for r in range(ntiles):
        cut = lambda a: np.ascontiguousarray(slabs.tile_slice(a, r, ntiles)).astype(dtype)
        o = O.Oracle(cfg, dtype)
        tiles.append(dict(o=o, f1=cut(fA), f2=cut(fB), R=[cut(a) for a in R], blank=cut(blank).astype(np.int32),
                          tau=np.full(cfg.sshape, 3.0 * np.float32(wl.kinevisc) + 0.5, dtype),
                          nb=slabs.neighbours(r, ntiles, wl.jbnd == 0)))
    uv = uvel.astype(dtype)
    for _ in range(steps):
        for t in tiles:
            t["o"].postcoll(t["f1"], t["tau"], *t["R"])
            t["o"].solids(t["f1"], t["blank"])
            t["o"].boundarycond(t["f1"], t["f2"], uv)
        planes = [(t["f1"][:, 1].copy(), t["f1"][:, ny].copy()) for t in tiles]
        for t in tiles:
            south, north = t["nb"]
            if south is not None:
                t["f1"][:, 0] = planes[south][1]
            if north is not None:
                t["f1"][:, ny + 1] = planes[north][0]
        for t in tiles:
            t["o"].drift(t["f2"], t["f1"])
            t["f1"], t["f2"] = t["f2"], t["f1"]
            t["o"].macrovars(*t["R"], t["f1"])
    return [(t["f1"], t["f2"], *t["R"]) for t in tiles]


def gpu_tiles(wl, ntiles, steps, storage="f32", kernel=None):
    from lbm_b200.slabs import SlabTile, step_local
    fA, fB, R, blank, uvel = global_start(wl)
    p = params_of(wl, iturb_pos=3, storage=storage)
    tiles = [SlabTile(p, r, ntiles) for r in range(ntiles)]
    for t in tiles:
        if kernel is not None:
            t.lbm.set_kernel(kernel)
        t.set_solids(cuda(blank.astype(np.int32)))
        t.set_inflow(cuda(uvel.astype(np.float32)))
        t.import_global(*(cuda(a.astype(np.float32)) for a in (fA, fB, *R)))
    step_local(tiles, steps)
    out = []
    for t in tiles:
        L = t.lbm
        f1, f2 = L.empty_f(), L.empty_f()
        L.state_export(f1, f2)
        M = [L.empty_s() for _ in range(4)]
        L.get_macro(*M)
        out.append(tuple(host(a) for a in (f1, f2, *M)))
        t.close()
    return out


@pytest.mark.parametrize("nl,ntiles,codes", [(19, 2, (1, 0, 12)), (27, 3, (1, 0, 12)), (19, 2, (11, 0, 22)),
                                             (27, 2, (1, 11, 22))])
def test_tiles_match_tiled_oracle(nl, ntiles, codes):
    ib, jb, kb = codes
    wl = W.Workload("slabs", 16, 12, 8, nl, steps=10, ibnd=ib, jbnd=jb, kbnd=kb, noise=3e-3, sphere=(6, 5, 4, 2))
    gpu = gpu_tiles(wl, ntiles, wl.steps)
    ref32 = oracle_tiles(wl, ntiles, np.float32, wl.steps)
    ref64 = oracle_tiles(wl, ntiles, np.float64, wl.steps)
    for r in range(ntiles):
        compare_to_floor(gpu[r], ref32[r], ref64[r], "tile %d of %d, codes %s" % (r, ntiles, codes))


@pytest.mark.parametrize("nl,storage", [(19, "f32"), (27, "f32"), (27, "f16")])
def test_tiles_equal_the_undivided_domain_with_periodic_k(nl, storage):
    """inflow i, periodic j and k: no boundary kernel reads a j ghost between the
    tile-local j copies and the exchange, so tiles and the whole domain agree
    (FP16 storage moves 16-bit planes)."""
    from lbm_b200 import Lbm
    wl = W.Workload("slabs", 16, 12, 8, nl, steps=12, ibnd=1, jbnd=0, kbnd=0, noise=3e-3, sphere=(6, 5, 4, 2))
    tiles = gpu_tiles(wl, 3, wl.steps, storage=storage)
    fA, fB, R, blank, uvel = global_start(wl)
    L = Lbm(params_of(wl, iturb_pos=3, storage=storage))
    L.set_solids(cuda(blank.astype(np.int32)))
    L.set_inflow(cuda(uvel.astype(np.float32)))
    L.state_import(*(cuda(a.astype(np.float32)) for a in (fA, fB, *R)))
    L.step(wl.steps)
    f1, f2 = L.empty_f(), L.empty_f()
    L.state_export(f1, f2)
    M = [L.empty_s() for _ in range(4)]
    L.get_macro(*M)
    whole = [host(a) for a in (f1, f2, *M)]
    L.close()
    ny = wl.ny // 3
    for r, t in enumerate(tiles):
        rows = slice(r * ny + 1, (r + 1) * ny + 1)
        for a, b in zip(t, whole):
            assert np.array_equal(a[1:-1, 1:-1, 1:-1], b[1:-1, rows, 1:-1]), r


@pytest.mark.parametrize("nl", [19, 27])
def test_fp16_tiles_in_the_folded_configuration(nl):
    """FP16-offset storage through the folded tiles (16-bit planes, x ghosts packed
    from the compact arrays): within the FP16 error budget of the FP32 tiles."""
    from tests.conftest import rel_l2
    wl = W.Workload("slabs", 16, 12, 8, nl, steps=10, ibnd=1, jbnd=0, kbnd=12, noise=3e-3, sphere=(6, 5, 4, 2))
    t32 = gpu_tiles(wl, 2, wl.steps, storage="f32")
    t16 = gpu_tiles(wl, 2, wl.steps, storage="f16")
    s = (slice(1, -1),) * 3
    for a, b in zip(t16, t32):
        assert np.all(np.isfinite(a[0]))
        assert rel_l2(a[2][s], b[2][s]) < 1e-4                                          # rho
        assert rel_l2(np.stack(a[3:])[(slice(None),) + s], np.stack(b[3:])[(slice(None),) + s]) < 1e-3   # u


def test_halo_switch_refusals():
    from lbm_b200 import Lbm, LbmError
    wl = W.Workload("slabs", 16, 12, 8, 19, steps=2)
    L = Lbm(params_of(wl, iturb_pos=3))
    with pytest.raises(LbmError, match="set_halo_j"):
        L.halo_pack_j(None, None)
    fA, fB, R, blank, uvel = global_start(wl)
    L.state_import(*(cuda(a.astype(np.float32)) for a in (fA, fB, *R)))
    with pytest.raises(LbmError, match="before the first import"):
        L.set_halo_j(True)
    L.close()


@pytest.mark.parametrize("nl,storage", [(19, "f32"), (27, "f16")])
def test_device_plane_layout_matches_the_host_mirror(nl, storage):
    """lbm_halo_pack_j writes the bytes lbm_b200.slabs.plane_from_ref describes
    (the layout the host-side exchange tests move between gloo ranks), and
    lbm_halo_plane_bytes equals slabs.plane_bytes."""
    from lbm_b200 import slabs
    from lbm_b200.slabs import SlabTile
    wl = W.Workload("slabs", 16, 12, 8, nl, steps=1, ibnd=1, jbnd=0, kbnd=12, noise=3e-3, sphere=(6, 5, 4, 2))
    fA, fB, R, blank, uvel = global_start(wl)
    t = SlabTile(params_of(wl, iturb_pos=3, storage=storage), 0, 2)
    assert t.lbm.halo_plane_bytes() == slabs.plane_bytes(wl.nx, wl.nz, nl, storage)
    f32 = [a.astype(np.float32) for a in (fA, fB, *R)]
    t.import_global(*(cuda(a) for a in f32))
    t.pack()
    tile_f1 = np.ascontiguousarray(slabs.tile_slice(f32[0], 0, 2))
    ny = wl.ny // 2
    assert np.array_equal(host(t.send[0]), slabs.plane_from_ref(tile_f1, 1, storage))     # plane j = 1, to the south
    assert np.array_equal(host(t.send[1]), slabs.plane_from_ref(tile_f1, ny, storage))    # plane j = ny, to the north
    t.close()
