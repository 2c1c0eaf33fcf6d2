"""Edge cases of the plain transport path (``pmo_run_plain``).

* Empty runs, ragged photon counts and split photon ranges: a photon's
  history depends only on (seed, photon id, optics), so any partition of the
  ids into ranges, and any launch shape, gives the same photons bit for bit
  and the same integer tallies (counters, fixed-point absorbed grid).
* The largest label table (255 labels with optics plus the end label).
* The smallest volume (one interior voxel).
* Error reporting: a photon over its event cap, and a photon entering a
  label without optical properties, end in a counted error that the host
  turns into ``PmoError`` with the matching status.  Neither touches memory
  outside the volume: the label table has 256 entries and every label
  indexes it.
"""
import numpy as np
import pytest
import torch

from pymonteopt_b200 import _abi as A
from pymonteopt_b200 import engine as E
from pymonteopt_b200._lib import PmoError
from pymonteopt_b200.problem import pencil_problem

pytestmark = pytest.mark.gpu


def _slab(nxy=23, nz=22):
    lab = np.ones((nxy, nxy, nz), np.uint8)
    lab[1:-1, 1:-1, 1:-1] = 0
    return pencil_problem(lab, 0.1, 1, [0.1], [10.0], [0.9], [1.37, 1.0])


def _spec(fluence=True):
    return E.TallySpec(nr=20, dr=0.1, fluence=A.PMO_FLU_GLOBAL if fluence else A.PMO_FLU_NONE,
                       export_exits=True, photon_stats=True)


def _per_photon(t):
    return (t.exit_add.cpu().numpy(), t.exit_p.cpu().numpy(), t.exit_v.cpu().numpy(),
            t.exit_w.cpu().numpy(), t.ph.cpu().numpy())


def _same_photons(a, b):
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_zero_photons_is_a_no_op(cuda):
    dp = E.DeviceProblem(_slab())
    t = E.run_plain(dp, 0, 1, spec=E.TallySpec(nr=20, dr=0.1, fluence=A.PMO_FLU_GLOBAL))
    torch.cuda.synchronize()
    t.check()
    assert not t.counters.any() and not t.ledger.any() and not t.absorbed.any()
    assert not t.rr.any()


@pytest.mark.parametrize("cuts", [(1,), (31, 33), (64, 65, 129), (1000, 1037)])
def test_photon_ranges_compose_bit_for_bit(cuda, cuts):
    dp = E.DeviceProblem(_slab())
    n, seed = 2111, 7
    whole = E.run_plain(dp, n, seed, spec=_spec())
    ref = _per_photon(whole)
    edges = [0, *cuts, n]
    absorbed = torch.zeros_like(whole.absorbed)
    counters = torch.zeros_like(whole.counters)
    for a, b in zip(edges[:-1], edges[1:]):
        part = E.run_plain(dp, b - a, seed, begin=a, spec=_spec())
        part.check()
        got = _per_photon(part)
        _same_photons([r[..., a:b] for r in ref], got)
        absorbed += part.absorbed
        counters += part.counters
    whole.check()
    assert torch.equal(absorbed, whole.absorbed)
    assert torch.equal(counters, whole.counters)


@pytest.mark.parametrize("threads,bps", [(32, 0), (512, 0), (128, 1), (96, 2)])
def test_launch_shape_does_not_change_photons(cuda, threads, bps):
    dp = E.DeviceProblem(_slab())
    n, seed = 5003, 11
    ref = E.run_plain(dp, n, seed, spec=_spec())
    got = E.run_plain(dp, n, seed, spec=_spec(), block_threads=threads, blocks_per_sm=bps)
    ref.check()
    got.check()
    _same_photons(_per_photon(ref), _per_photon(got))
    assert torch.equal(ref.counters, got.counters)
    assert torch.equal(ref.absorbed, got.absorbed)
    # FP64 sums in another order: equal to rounding
    np.testing.assert_allclose(got.ledger.cpu().numpy(), ref.ledger.cpu().numpy(),
                               rtol=1e-12, atol=1e-12)


def test_full_label_table(cuda):
    """255 labels with their own optics and refractive indices, one end label."""
    rng = np.random.default_rng(3)
    nl = 255
    lab = np.full((34, 34, 34), nl, np.uint8)
    lab[1:-1, 1:-1, 1:-1] = rng.integers(0, nl, (32, 32, 32), dtype=np.uint8)
    ma = rng.uniform(0.01, 0.5, nl)
    ms = rng.uniform(1.0, 20.0, nl)
    g = rng.uniform(0.0, 0.95, nl)
    n = np.concatenate([rng.uniform(1.0, 1.6, nl), [1.0]])
    prob = pencil_problem(lab, 0.05, nl, ma, ms, g, n)
    dp = E.DeviceProblem(prob)
    t = E.run_plain(dp, 20000, 5, spec=E.TallySpec(nr=20, dr=0.05))
    torch.cuda.synchronize()
    t.check()
    L = t.ledger.cpu().numpy()
    inflow = L[A.PMO_L_WINIT] + L[A.PMO_L_RGAIN]
    outflow = (L[A.PMO_L_RD] - L[A.PMO_L_SPEC] + L[A.PMO_L_TT] + L[A.PMO_L_EXIT0] +
               L[A.PMO_L_ABS] + L[A.PMO_L_RLOSS] + L[A.PMO_L_ERRW])
    assert abs(inflow - outflow) <= 1e-6 * inflow
    c = t.host_counters()
    assert c[A.PMO_C_PHOTONS] == 20000 and c[A.PMO_C_FRESNEL] > 0


def test_one_voxel_volume(cuda):
    lab = np.ones((3, 3, 3), np.uint8)
    lab[1, 1, 1] = 0
    prob = pencil_problem(lab, 0.1, 1, [0.5], [20.0], [0.8], [1.4, 1.0])
    dp = E.DeviceProblem(prob)
    t = E.run_plain(dp, 10000, 2, spec=E.TallySpec(nr=4, dr=0.05, fluence=A.PMO_FLU_GLOBAL))
    torch.cuda.synchronize()
    t.check()
    s = t.summary()
    assert s["counters"][A.PMO_C_PHOTONS] == 10000
    assert 0.0 < s["A"] < 1.0 and s["Rd"] > 0.0
    # all absorption lands in the single interior voxel
    w = E.absorbed_weight(t).cpu().numpy()
    assert w[1, 1, 1] > 0 and np.count_nonzero(w) == 1
    # fixed-point deposits against the FP64 ledger: rounding of 2^-33 at most per deposit
    assert w[1, 1, 1] == pytest.approx(s["A"] * 10000, rel=1e-7)


def test_event_cap_is_reported(cuda):
    dp = E.DeviceProblem(_slab())
    t = E.run_plain(dp, 1000, 3, spec=E.TallySpec(nr=20, dr=0.1), max_events=5)
    torch.cuda.synchronize()
    with pytest.raises(PmoError) as err:
        t.check()
    assert err.value.status == A.PMO_ERR_STEP_CAP
    c = t.host_counters()
    assert c[A.PMO_C_ERR_CAP] > 0 and c[A.PMO_C_PHOTONS] == 1000
    # the weight of the stopped photons is booked, so the ledger still closes
    assert t.ledger.cpu().numpy()[A.PMO_L_ERRW] > 0


def test_label_without_optics_is_reported(cuda):
    prob = _slab()
    dp = E.DeviceProblem(prob)
    # a label past the table's defined entries, placed in the beam's path
    cx, cy = prob.center
    dp.labels[cx, cy, 4] = 200
    dp.build_words()
    t = E.run_plain(dp, 1000, 4, spec=E.TallySpec(nr=20, dr=0.1))
    torch.cuda.synchronize()
    with pytest.raises(PmoError) as err:
        t.check()
    assert err.value.status == A.PMO_ERR_LABEL
    assert t.host_counters()[A.PMO_C_ERR_LABEL] > 0


def test_model_start_sees_in_place_volume_edit(cuda):
    """start() uploads the labels again and compares them with the resident
    copy on the device: an in-place edit of model.voxel_model between two
    starts takes effect (box map rebuilt), an unchanged volume stays."""
    from pymonteopt_b200 import VoxelPlateModel
    m = VoxelPlateModel(nPh=50000, keep_exits=False, verbose=False, device=cuda)
    m.build(x_size=3.0, y_size=3.0, voxel_space=0.1, thickness=[0.5, 1.0], n=[1.4, 1.4],
            n_air=1.0, ma=[0.1, 2.0], ms=[10.0, 10.0], g=[0.9, 0.9])
    rd0 = m.start(5).getRdTtValues()["Rd"]
    dp0 = m._dprob
    assert m.start(5).getRdTtValues()["Rd"] == rd0 and m._dprob is dp0
    # turn the strongly absorbing second layer into the first layer's tissue
    vm = m.model.voxel_model
    vm[vm == 1] = 0
    rd1 = m.start(5).getRdTtValues()["Rd"]
    assert m._dprob is dp0 and rd1 > rd0 + 0.01, (rd0, rd1)
    lab = m._dprob.labels.cpu().numpy()
    assert np.array_equal(lab, vm.view(np.uint8))
    words = m._dprob.words.cpu().numpy().view(np.uint16)
    assert np.array_equal(words & 0xff, lab)


def test_volume_checks_run_on_the_device_copy(cuda):
    """The shell and label-range checks run on the uploaded labels: a broken
    shell or a label without optics is refused with the host check's message,
    both when a problem is uploaded and when start() finds an edited volume."""
    from pymonteopt_b200 import VoxelPlateModel
    good = _slab()
    E.DeviceProblem(good)
    for edit, msg in (((0, 5, 5), "shell"), ((5, 5, 5), "no optical properties")):
        lab = good.labels.copy()
        lab[edit] = 0 if msg == "shell" else 7
        bad = pencil_problem(lab, 0.1, 1, [0.1], [10.0], [0.9], [1.37, 1.0])
        with pytest.raises(ValueError, match=msg):
            bad.validate()                       # host form of the same checks
        with pytest.raises(ValueError, match=msg):
            E.DeviceProblem(bad)
    m = VoxelPlateModel(nPh=1000, keep_exits=False, verbose=False, device=cuda)
    m.build(x_size=2.0, y_size=2.0, voxel_space=0.1, thickness=[1.0], n=[1.4], n_air=1.0,
            ma=[0.1], ms=[10.0], g=[0.9])
    m.start(1)
    m.model.voxel_model[0, 3, 3] = 0
    with pytest.raises(ValueError, match="shell"):
        m.start(1)


def test_plate_volume_is_page_locked_and_exact(cuda):
    """With a GPU present a plate volume is built in page-locked memory (the
    upload is then a direct copy); its bytes are still the reference's
    layer-by-layer fill, on a first build and on a rebuild of the same size
    (a reused block)."""
    from pymonteopt_b200 import voxel as VX
    params = dict(x_size=3.1, y_size=2.7, voxel_space=0.1, thickness=[0.2, 0.9, 0.4],
                  n=[1.4, 1.37, 1.45], n_air=1.0, ma=[0.1, 0.2, 0.3], ms=[10, 20, 30],
                  g=[0.9, 0.8, 0.7])
    m = VX.PlateModel()
    m.verbose = False
    m.set_params(**params)
    for _ in range(2):
        m.build()
        vm = m.voxel_model
        assert torch.from_numpy(vm).is_pinned()
        ref = np.zeros(vm.shape, np.int8)
        ref[:, :, 1:3], ref[:, :, 3:12], ref[:, :, 12:16] = 0, 1, 2
        ref[0] = ref[-1] = 3
        ref[:, 0] = ref[:, -1] = 3
        ref[:, :, 0] = ref[:, :, -1] = 3
        assert vm.shape == (33, 29, 17) and np.array_equal(vm, ref)
