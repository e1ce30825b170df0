"""Project-input mirror (blaze.project) against the reference's own parser
and header layouts, compiled on the host (oracle/_ref)."""
import ctypes as C
import os

import numpy as np
import pytest

import bindings
import canon
from blaze import types as T
from blaze.project import Project, read_state_file

from conftest import REFERENCE

REF_PROJECTS = os.path.join(REFERENCE, "Projects")
need_ref_tree = pytest.mark.skipif(not os.path.isdir(REF_PROJECTS),
                                   reason="reference project tree not present")
need_ref_lib = pytest.mark.skipif(not bindings.ref_available(), reason="oracle/_ref not built")
need_ref_parse = pytest.mark.skipif(
    not os.path.isfile(os.path.join(os.path.dirname(bindings.REF_SO), "refparse")),
    reason="oracle/_ref/refparse not built")


@need_ref_lib
def test_struct_layouts_match_reference_headers():
    R = bindings.RefHost()
    for name, typ in T.BOUNDARY_TYPES.items():
        assert C.sizeof(typ) == R.sizeof(name), name


@need_ref_lib
@need_ref_tree
@pytest.mark.parametrize("project,world", [("1.Particles_Box", "Spheres_128cm"),
                                           ("2.Silo", "SPH_90"), ("3.BallMill", "Mill_SPH30")])
def test_parser_matches_reference(project, world):
    R = bindings.RefHost()
    rp, w, p, d = R.parse(REF_PROJECTS, project, world)
    P = Project.load(REF_PROJECTS, project, world)
    assert (rp.n_w, rp.n_p, rp.n_d, rp.num_particles) == (P.n_w, P.n_p, P.n_d, P.num_particles)
    for i in range(rp.n_w):
        assert canon.wobj(w[i]) == canon.wobj(P.wobj[i])
    for i in range(rp.n_p):
        assert canon.pobj_sphere(p[i], rp.n_p) == canon.pobj_sphere(P.pobj[i], P.n_p)
    for i in range(rp.n_d):
        assert canon.dobj(d[i]) == canon.dobj(P.dobj[i])
    assert np.float32(rp.delta_t) == P.delta_t
    assert (rp.grid_size.x, rp.grid_size.y, rp.grid_size.z) == tuple(float(v) for v in P.grid_size)



@need_ref_parse
@need_ref_tree
@pytest.mark.parametrize("project,world", [("1.Particles_Box", "Poly_128cm"),
                                           ("4.UnitTests", "2P")])
def test_polyhedron_parser_matches_reference(project, world):
    """ReadPObject_Poly: the dodecahedron (Format 1: offset vertices,
    comma-separated faces) and the cube (Format 0), field by field; the
    run setup's inertia scaling (main.cpp:622-626) on top of the parser's
    inverted tensor."""
    rp, w, p, d = bindings.RefHost.parse_isolated(REF_PROJECTS, project, world)
    P = Project.load(REF_PROJECTS, project, world)
    assert P.particle_type == 1 and rp.particle_type == 1
    for i in range(rp.n_p):
        ref = p[i]
        mine = T.POBJ.from_buffer_copy(bytes(P.pobj[i]))
        scale = np.float32(np.float32(1.0) / np.float32(np.float32(np.float32(
            np.float32(0.4) * np.float32(ref.radius)) * np.float32(ref.radius)) *
            np.float32(ref.mass)))
        for g in range(9):
            expect = np.float32(scale * np.float32(ref.InertiaT[g]))
            assert np.float32(mine.InertiaT[g]) == expect, (i, g)
            mine.InertiaT[g] = ref.InertiaT[g]
        assert canon.pobj_poly(ref, rp.n_p) == canon.pobj_poly(mine, P.n_p), i
    for i in range(rp.n_w):
        assert canon.wobj(w[i]) == canon.wobj(P.wobj[i])

@need_ref_tree
def test_state_file_spec4_silo():
    P = Project.load(REF_PROJECTS, "2.Silo", "SPH_90")
    st = P.read_state()
    assert st["spec_type"] == 4
    assert st["pos"].shape == (1950, 3)
    assert st["pid"][0] == 0 and st["pid"][1] == 130
    np.testing.assert_allclose(st["pos"][0], [0.399982, 30.4, 0.400001], rtol=1e-6)


def test_synthetic_box_project(tmp_path):
    from blaze import synth
    P, st = synth.box_project(str(tmp_path))
    assert P.num_particles == 10000
    si = P.sim_info
    assert (si.num_NNCells.x, si.num_NNCells.y, si.num_NNCells.z) == (52, 52, 52)
    # face normals point into the box
    for s in range(6):
        S = P.wobj[0].surfaces[s]
        n = np.array([S.normal.x, S.normal.y, S.normal.z])
        c = np.array([S.centroid.x, S.centroid.y, S.centroid.z])
        assert np.dot(n, np.array([5.0, 5.0, 5.0]) - c) > 0
    # KN mode, same type: Cn from COR with the 0.03808 correction and m/2
    import math
    m = np.float32(P.pobj[0].mass)
    cor = 0.5 - 0.03808
    L = math.log(cor)
    cn = -2.0 * L * math.sqrt(1e5 * float(m) / 2) / math.sqrt(L * L + math.pi ** 2)
    assert abs(P.pobj[0].PP[0].Cn - cn) / cn < 1e-6
    assert abs(P.pobj[0].InertiaT[0] - 1.0 / (0.4 * 0.1 * 0.1 * float(m))) / P.pobj[0].InertiaT[0] < 1e-6


def test_project_errors(tmp_path):
    from blaze.project import ProjectError
    with pytest.raises(ProjectError):
        Project.load(str(tmp_path), "missing", "nothing")
