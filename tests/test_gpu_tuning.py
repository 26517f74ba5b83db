"""GPU checks of the launch-shape knobs: every filter k-tile width (and the per-thread register
kernel where it applies) gives the same energy, forces and stress to rounding, for many-species
and few-species boxes, in float64 and in the mixed form."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

KW = dict(method="spme", mesh_spacing=1.2, interpolation_nodes=5, c6tol=1.0, r_cut=6.0)


@pytest.mark.parametrize("precision,z_max,n", [("fp64", 54, 160), ("mixed", 54, 160), ("fp64", 8, 120),
                                               ("mixed", 8, 120)])
def test_filter_tiles_agree(precision, z_max, n, cuda_device):
    from fourierd3_b200 import D3Model, structures as st

    pos, cell, z = st.random_box(41, n, z_max=z_max)
    m = D3Model(z, cell, precision=precision, device=cuda_device, **KW)
    e0, f0, s0 = (t.clone() for t in m(pos, cell))
    tol_e = 1e-12 if precision == "fp64" else 2e-6
    tol_f = 1e-10 if precision == "fp64" else 1e-5
    tried = []
    for kt in (0, 1, 2, 4, 8, 16):
        try:
            m.engine.set_tuning(filter_kt=kt)
        except ValueError:
            # the register kernel takes at most 8 species; wide float64 tiles outgrow shared memory
            assert (kt == 0 and len(np.unique(z)) > 8) or (kt >= 8 and precision == "fp64")
            continue
        assert m.engine.tuning()["filter_kt"] == kt
        e, f, s = m(pos, cell)
        assert abs(float(e) - float(e0)) <= tol_e * abs(float(e0)), (kt, float(e), float(e0))
        assert (f - f0).abs().max().item() <= tol_f, kt
        assert (s - s0).abs().max().item() <= tol_f, kt
        tried.append(kt)
    assert len(tried) >= 3


def test_bad_tile_rejected(cuda_device):
    from fourierd3_b200 import D3Model, structures as st

    pos, cell, z = st.random_box(42, 60, z_max=54)
    m = D3Model(z, cell, precision="mixed", device=cuda_device, **KW)
    with pytest.raises(ValueError):
        m.engine.set_tuning(filter_kt=3)
    with pytest.raises(ValueError):
        m.engine.set_tuning(filter_kt=0)    # register kernel: at most 8 species


def test_autotune_filter_sets_a_valid_tile(cuda_device):
    from fourierd3_b200.batch import D3Batch, autotune_filter
    from fourierd3_b200 import structures as st

    structs = [st.random_box(50 + k, 40 + 30 * k, z_max=54 if k % 2 else 6) for k in range(4)]
    b = D3Batch(structs, precision="mixed", device=cuda_device, **KW)
    e0 = b()[0].clone()
    res = autotune_filter(b, reps=1)
    assert res
    for c, (best, times) in res.items():
        assert best in times
    e1 = b()[0]
    assert torch.allclose(e0, e1, rtol=2e-6, atol=0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_spread_column_chunks_agree(precision, cuda_device):
    """Per-tile spread (zc = 0) against column chunks of several lengths, and the per-tile staging
    fallback of a column chunk that exceeds its staging cap (all oxygen atoms of the 648-atom box
    fall into one 16x16 column of a 16^3 mesh)."""
    from fourierd3_b200 import D3Model, structures as st

    tol_e = 1e-12 if precision == "fp64" else 2e-6
    tol_f = 1e-10 if precision == "fp64" else 1e-5
    for kw, zcs in ((KW, (1, 3, 8)), (dict(KW, mesh_spacing=4.8), (1, 2))):
        pos, cell, z = st.sio2_box(0)
        m = D3Model(z, cell, precision=precision, device=cuda_device, **kw)
        m.engine.set_tuning(spread_zc=0)
        e0, f0, s0 = (t.clone() for t in m(pos, cell))
        for zc in zcs:
            for cap in (0, 256):
                m.engine.set_tuning(spread_zc=zc, spread_cap=cap)
                assert m.engine.tuning()["spread_zc"] == zc   # the column kernel runs
                e, f, s = m(pos, cell)
                assert abs(float(e) - float(e0)) <= tol_e * abs(float(e0)), (zc, cap)
                assert (f - f0).abs().max().item() <= tol_f, (zc, cap)
                assert (s - s0).abs().max().item() <= tol_f, (zc, cap)
    with pytest.raises(ValueError):
        m.engine.set_tuning(spread_cap=100)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_x_pass_agrees_with_3d_fft(precision, cuda_device):
    """cuFFT (y, z) planes + the fused x-FFT / filter / inverse x-FFT kernel against 3D cuFFT
    around the separate filter, for SPME and PME, one to four species, nx = 64 and 128, and
    pencils of 1, 2 and 4 kz values (float pencils of 2 and 4 move as 16-byte pairs, shifted by
    one kz on the rows of odd parity; the case meshes have odd nz/2 + 1)."""
    import golden_cases as gc
    from fourierd3_b200 import D3Model

    tol_e = 1e-12 if precision == "fp64" else 2e-6
    tol_f = 1e-10 if precision == "fp64" else 1e-5
    ran = 0
    for name in ("sio2_648_spme_p5", "sio2_648_pme_p5", "hcno_240_spme_p6", "hcno_240_spme_p4_tol1e-4"):
        rec = gc.load(name)
        m = D3Model(rec["numbers"], rec["cell"], precision=precision, device=cuda_device,
                    **gc.model_kwargs(rec["config"]))
        m.engine.set_tuning(fft_x=0)
        assert m.engine.tuning()["fft_x"] == 0
        e0, f0, s0 = (t.clone() for t in m(rec["positions"], rec["cell"]))
        m.engine.set_tuning(fft_x=1)
        if m.engine.tuning()["fft_x"] != 1:
            continue   # more than 4 species or 8 ranks, or an nx outside 64/128/256
        ran += 1
        for kz in (-1, 1, 2, 4):
            m.engine.set_tuning(xpencil=kz)
            got = m.engine.tuning()["xpencil"]
            assert got in (1, 2, 4) and (kz == -1 or got <= kz), (name, kz, got)   # wider than shared memory: default
            e, f, s = m(rec["positions"], rec["cell"])
            assert abs(float(e) - float(e0)) <= tol_e * abs(float(e0)), (name, kz, float(e), float(e0))
            assert (f - f0).abs().max().item() <= tol_f, (name, kz)
            assert (s - s0).abs().max().item() <= tol_f, (name, kz)
    assert ran >= 2
    with pytest.raises(ValueError):
        m.engine.set_tuning(xpencil=3)


def test_tma_x_pass_agrees_with_3d_fft(cuda_device):
    """The TMA-moved fused x-pass (mixed precision) against 3D cuFFT around the separate filter,
    for SPME and PME, one to four species, nx = 64 and 128, units of 8, 16 and 32 flattened
    (y, kz) values and of one or two ranks (an odd rank count leaves a padded last group)."""
    import golden_cases as gc
    from fourierd3_b200 import D3Model

    ran = 0
    for name in ("sio2_648_spme_p5", "sio2_648_pme_p5", "hcno_240_spme_p6", "hcno_240_spme_p4_tol1e-4",
                 "tiny_6_spme_p4"):
        rec = gc.load(name)
        m = D3Model(rec["numbers"], rec["cell"], precision="mixed", device=cuda_device,
                    **gc.model_kwargs(rec["config"]))
        m.engine.set_tuning(fft_x=0)
        e0, f0, s0 = (t.clone() for t in m(rec["positions"], rec["cell"]))
        for xq in (8, 16, 32):
            for xr in (1, 2):
                m.engine.set_tuning(fft_x=2, xq=xq, xranks=xr)
                t = m.engine.tuning()
                if t["fft_x"] != 2:
                    continue   # nx outside 64/128/256, more than 4 species, or the unit does not fit twice
                assert (t["xq"], t["xranks"]) == (xq, xr)
                ran += 1
                e, f, s = m(rec["positions"], rec["cell"])
                assert abs(float(e) - float(e0)) <= 2e-6 * abs(float(e0)), (name, xq, xr, float(e), float(e0))
                assert (f - f0).abs().max().item() <= 1e-5, (name, xq, xr)
                assert (s - s0).abs().max().item() <= 1e-5, (name, xq, xr)
        m.engine.set_tuning(fft_x=2, xq=-1, xranks=-1)
    assert ran >= 12
    with pytest.raises(ValueError):
        m.engine.set_tuning(xq=12)
    with pytest.raises(ValueError):
        m.engine.set_tuning(xranks=3)


def test_tma_x_pass_float64_plan_keeps_its_path(cuda_device):
    """fft_x = 2 is a mixed-precision path; a float64 plan reports the path it actually runs."""
    import golden_cases as gc
    from fourierd3_b200 import D3Model

    rec = gc.load("sio2_648_spme_p5")
    m = D3Model(rec["numbers"], rec["cell"], precision="fp64", device=cuda_device, **gc.model_kwargs(rec["config"]))
    m.engine.set_tuning(fft_x=2)
    t = m.engine.tuning()
    assert t["fft_x"] == 0 and t["xq"] == 0
    e, f, s = m(rec["positions"], rec["cell"])
    assert abs(float(e) - float(rec["energy_ev"])) <= 1e-10 * abs(float(rec["energy_ev"]))


def test_autotune_fft_x_picks_a_timed_path(cuda_device):
    """batch.autotune_fft_x times the 3D path and the fused x-pass at each pencil width on the
    plan's heaviest structure, leaves the fastest set on the plan, and the batch results agree
    with the 3D path (few species: the fused path applies; many species: it does not)."""
    from fourierd3_b200 import structures as st
    from fourierd3_b200.batch import D3Batch, autotune_fft_x

    structs = [st.sio2_box(0), st.random_box(61, 90, z_max=54)]
    b = D3Batch(structs, precision="mixed", device=cuda_device, **KW)
    e0 = b()[0].clone()
    res = autotune_fft_x(b, reps=1)
    assert len(res) == 2
    for n, (best, times) in res.items():
        assert best == min(times, key=times.get) and "0" in times
        eng = list(b._engines.values())[n]
        t = eng.tuning()
        parts = best.split("/")
        if best == "0":
            assert t["fft_x"] == 0
        elif parts[0] == "1":
            assert t["fft_x"] == 1 and t["xpencil"] == int(parts[1])
        else:
            assert t["fft_x"] == 2 and (t["xq"], t["xranks"]) == (int(parts[1]), int(parts[2]))
    fused = [times for _, times in res.values() if len(times) > 1]
    # SiO2: 64^3, 2 species, rank 4 (both fused kernels apply); the 54-species box: neither
    assert len(fused) == 1 and {"0", "1/1", "1/2", "1/4"} <= set(fused[0])
    assert any(k.startswith("2/") for k in fused[0])
    e = b()[0]
    assert torch.allclose(e, e0, rtol=2e-6, atol=0.0)


@pytest.mark.parametrize("z_max,n,seed", [(54, 300, 61), (43, 200, 62), (12, 160, 63), (6, 120, 64)])
def test_tensor_core_filter_agrees(z_max, n, seed, cuda_device):
    """Mixed form: the tcgen05 filter (tf32 high/low split, three products per k-point) against
    the CUDA-core filter on the same plan -- energy 2e-6 relative, forces and stress 1e-5 --
    for 6 to 54 species (ranks 3 to 8, so padded columns of the 16-wide product as well)."""
    from fourierd3_b200 import D3Model, structures as st

    pos, cell, z = st.random_box(seed, n, z_max=z_max, angles=(75.0, 105.0))
    m = D3Model(z, cell, precision="mixed", device=cuda_device, **KW)
    m.engine.set_tuning(filter_mma=0)
    assert m.engine.tuning()["filter_mma"] == 0
    e0, f0, s0 = (t.clone() for t in m(pos, cell))
    m.engine.set_tuning(filter_mma=1)
    assert m.engine.tuning()["filter_mma"] == 1
    e, f, s = m(pos, cell)
    assert torch.isfinite(e).item()
    assert abs(float(e) - float(e0)) <= 2e-6 * abs(float(e0)), (float(e), float(e0))
    assert (f - f0).abs().max().item() <= 1e-5
    assert (s - s0).abs().max().item() <= 1e-5
    e2, f2, s2 = m(pos, cell)                 # repeat: bitwise equal
    assert float(e2) == float(e) and torch.equal(f2, f) and torch.equal(s2, s)


def test_tensor_core_filter_default_and_bounds(cuda_device):
    """Default: CUDA cores; the tensor-core filter is in effect only where asked for and where it
    applies (mixed precision, at most 64 species and 8 ranks); out-of-range values are rejected."""
    from fourierd3_b200 import D3Model, structures as st

    pos, cell, z = st.random_box(65, 120, z_max=20)
    m = D3Model(z, cell, precision="mixed", device=cuda_device, **KW)
    assert m.engine.tuning()["filter_mma"] == 0
    m.engine.set_tuning(filter_mma=1)
    assert m.engine.tuning()["filter_mma"] == 1
    with pytest.raises(ValueError):
        m.engine.set_tuning(filter_mma=2)
    m64 = D3Model(z, cell, precision="fp64", device=cuda_device, **KW)
    m64.engine.set_tuning(filter_mma=1)
    assert m64.engine.tuning()["filter_mma"] == 0          # float64 stays on CUDA cores


@pytest.mark.parametrize("precision,case,applies", [("mixed", "sio2", True), ("fp64", "hhe", True),
                                                    ("mixed", "small_mesh", True), ("mixed", "pme_p6", True),
                                                    ("fp64", "sio2", False), ("mixed", "many", False)])
def test_tile_gather_agrees_with_per_atom_gather(precision, case, applies, cuda_device):
    """The tile-staged gather (one CTA per (mesh tile, species), the tile's potential box staged
    once: TMA for interior tiles, wrapped plain loads for tiles at the upper mesh edge and for
    meshes narrower than the box) gives the per-atom gather's energy, forces and stress to
    rounding. Cases: the 648-atom SiO2 box (64^3, rank 4); H/He in float64 (rank 3, 32^3); a
    16^3 mesh narrower than the 20-point box (rank 5, every box wraps); PME p=6 (21 x 21 x 16
    box, rank 4); and two where the box outgrows shared memory (float64 rank 4, 53 species rank
    8), which keep the per-atom gather."""
    from fourierd3_b200 import D3Model, structures as st

    kw = dict(KW)
    if case == "sio2":
        pos, cell, z = st.sio2_box(0)
    elif case == "hhe":
        pos, cell, z = st.random_box(73, 150, z_max=2, density=(1.0, 1.5))
        kw["mesh_spacing"] = 0.6
    elif case == "many":
        pos, cell, z = st.random_box(71, 200, z_max=54)
    elif case == "small_mesh":
        pos, cell, z = st.random_box(72, 60, z_max=8, density=(2.0, 2.0))
        kw["mesh_spacing"] = 2.0
    else:
        pos, cell, z = st.random_box(73, 150, z_max=4, density=(1.0, 1.5))
        kw.update(method="pme", interpolation_nodes=6)
    m = D3Model(z, cell, precision=precision, device=cuda_device, **kw)
    m.engine.set_tuning(gather_tile=0)
    assert m.engine.tuning()["gather_tile"] == 0
    e0, f0, s0 = (t.clone() for t in m(pos, cell))
    m.engine.set_tuning(gather_tile=1)
    assert (m.engine.tuning()["gather_tile"] == 1) == applies, m.engine.tuning()
    e, f, s = m(pos, cell)
    tol_e = 1e-13 if precision == "fp64" else 1e-6
    tol_f = 1e-11 if precision == "fp64" else 2e-5
    assert abs(float(e) - float(e0)) <= tol_e * abs(float(e0)), (float(e), float(e0))
    assert (f - f0).abs().max().item() <= tol_f
    assert (s - s0).abs().max().item() <= tol_f
    # repeat: the tile gather is deterministic (no atomics)
    e2, f2, s2 = m(pos, cell)
    assert float(e2) == float(e) and torch.equal(f2, f) and torch.equal(s2, s)


def test_tile_gather_knob_bounds(cuda_device):
    from fourierd3_b200 import D3Model, structures as st

    pos, cell, z = st.sio2_box(0)
    m = D3Model(z, cell, precision="mixed", device=cuda_device, **KW)
    assert m.engine.tuning()["gather_tile"] == 0        # the default: the per-atom gather
    m.engine.set_tuning(gather_tile=1)
    assert m.engine.tuning()["gather_tile"] == 1
    m.engine.set_tuning(gather_tile=-1)
    assert m.engine.tuning()["gather_tile"] == 0
    with pytest.raises(ValueError):
        m.engine.set_tuning(gather_tile=2)


@pytest.mark.parametrize("fft_x,variant", [(2, 1), (2, 2), (1, 2)])
def test_fused_yz_transforms_agree_with_cufft(fft_x, variant, cuda_device):
    """The fused (y, z) plane transforms (clusters of 2 or 4 CTAs sharing each 256 x 256 plane
    through distributed shared memory, one pass over the mesh each way) give cuFFT's energy,
    forces and stress to float rounding, under the TMA x-pass (fft_x=2, the benchmarked knobs)
    and the cp.async x-pass (fft_x=1): the 41,472-atom SiO2 replica, 256^3 mesh, mixed precision.
    The energy is checked against the float64 form as well, at the mixed form's tolerance."""
    from fourierd3_b200 import D3Model, structures as st

    pos, cell, z = st.sio2_scaled(4)
    m = D3Model(z, cell, precision="mixed", device=cuda_device, **KW)
    knobs = dict(fft_x=2, xq=4, xranks=4) if fft_x == 2 else dict(fft_x=1)
    m.engine.set_tuning(**knobs)
    assert m.engine.tuning()["fft_yz"] == 1            # the default where it applies
    m.engine.set_tuning(fft_yz=0)
    assert m.engine.tuning()["fft_yz"] == 0
    e0, f0, s0 = (t.clone() for t in m(pos, cell))
    m.engine.set_tuning(fft_yz=variant)
    assert m.engine.tuning()["fft_yz"] == variant
    e, f, s = m(pos, cell)
    assert abs(float(e) - float(e0)) <= 2e-7 * abs(float(e0)), (float(e), float(e0))
    assert (f - f0).abs().max().item() <= 5e-6
    assert (s - s0).abs().max().item() <= 5e-8
    m64 = D3Model(z, cell, precision="fp64", device=cuda_device, **KW)
    e64, f64, s64 = m64(pos, cell)
    assert abs(float(e) - float(e64)) <= 1e-6 * abs(float(e64))
    assert (f - f64).abs().max().item() <= 1e-4
    # deterministic: no atomics in either transform
    e2, f2, s2 = m(pos, cell)
    assert float(e2) == float(e) and torch.equal(f2, f) and torch.equal(s2, s)


def test_fused_yz_transforms_non_cubic_mesh(cuda_device):
    """A 50 x 80 x 80 A box at h = 1.2 A: a 128 x 256 x 256 mesh (nx = 128 planes of 256 x 256,
    the nx = 128 TMA x-pass on the padded spectrum), 3,000 random atoms of 4 elements, mixed
    precision: the fused (y, z) transforms against cuFFT's, and against the float64 form."""
    from fourierd3_b200 import D3Model

    rng = np.random.default_rng(11)
    cell = np.diag([50.0, 80.0, 80.0])
    n = 3000
    frac = rng.random((n, 3))
    pos = frac @ cell
    z = rng.choice([1, 6, 7, 8], size=n)
    m = D3Model(z, cell, precision="mixed", device=cuda_device, **KW)
    assert tuple(m.mesh) == (128, 256, 256)
    m.engine.set_tuning(fft_x=2, xq=4, xranks=min(4, m.setup.n_rank) if m.setup.n_rank in (1, 2, 4) else 1)
    for variant in (1, 2):
        m.engine.set_tuning(fft_yz=0)
        e0, f0, s0 = (t.clone() for t in m(pos, cell))
        m.engine.set_tuning(fft_yz=variant)
        assert m.engine.tuning()["fft_yz"] == variant, m.engine.tuning()
        e, f, s = m(pos, cell)
        assert abs(float(e) - float(e0)) <= 2e-7 * abs(float(e0)), (variant, float(e), float(e0))
        assert (f - f0).abs().max().item() <= 5e-6
        assert (s - s0).abs().max().item() <= 5e-8
    m64 = D3Model(z, cell, precision="fp64", device=cuda_device, **KW)
    e64, f64, _ = m64(pos, cell)
    assert abs(float(e) - float(e64)) <= 1e-6 * abs(float(e64))
    assert (f - f64).abs().max().item() <= 1e-4


def test_fused_yz_transforms_where_they_apply(cuda_device):
    """In effect only with the x-pass, mixed precision and a 256 x 256 (y, z) plane."""
    from fourierd3_b200 import D3Model, structures as st

    pos, cell, z = st.sio2_box(0)                      # 64^3 mesh
    m = D3Model(z, cell, precision="mixed", device=cuda_device, **KW)
    m.engine.set_tuning(fft_yz=1, fft_x=2)
    assert m.engine.tuning()["fft_yz"] == 0
    with pytest.raises(ValueError):
        m.engine.set_tuning(fft_yz=3)
