"""The contracted particle-particle law (blaze_options.fast_law = 1) against
the reference's own kernels on its own project (oracle-A golden fixture:
Projects/2.Silo world SPH_90, 1,950 spheres with the silo hatch), and
against the FP64 restatement of the reference law on 20,000 spheres of
the synthetic silo workload settled into contact.  (A run with energy tallies, such as
the ball-mill fixture, keeps the reference's arithmetic in the law.)

Bar: the contact lists are the reference's bit for bit (the contact test is
not contracted); the forces of the first step agree within 1e-5 relative,
per particle, where the scale of a particle is the larger of its net force
and its weight (a particle whose contact forces nearly cancel carries their
rounding, not its net force's); the state after the step agrees within the
same relative bound on the velocity change.  The error of the bit-exact law
against FP64 is printed beside the contracted one's."""
import numpy as np
import pytest

from bindings import Restated
from blaze import device, synth
from conftest import Golden

pytestmark = pytest.mark.gpu

TOL = 1e-5


def gpu_sim(g, **opts):
    s = device.Simulation(sim_info=g.sim_info, wobj=g.wobj, n_w=g.n_w, pobj=g.pobj, n_p=g.n_p,
                          dobj=g.dobj, n_d=g.n_d, **opts)
    s.set_cylinder_rotation(g.cyl_rot)
    st = g.init()
    s.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    return s


def rel_err(f, ref, weight):
    scale = np.maximum(np.linalg.norm(ref, axis=1), weight)
    return float((np.linalg.norm(f.astype(np.float64) - ref, axis=1) / scale).max())


@pytest.mark.parametrize("name", ["silo_sph90"])
def test_fast_law_vs_reference_kernels(name):
    g = Golden(name)
    s = gpu_sim(g, capture_forces=1, fast_law=1)
    s.step(1)
    ref = g.at(1)
    st = s.state()
    assert st["status"] == 0, device.decode_status(st["status"])
    nn, lst = s.nlist()
    np.testing.assert_array_equal(nn, ref["nn"])
    w = ref["list"].shape[1]
    np.testing.assert_array_equal(lst[:, :w], ref["list"])
    np.testing.assert_array_equal(st["pid"], ref["pid"])
    f = s.forces()
    gmag = float(np.linalg.norm([g.sim_info.Force_Field.x, g.sim_info.Force_Field.y,
                                 g.sim_info.Force_Field.z]))
    mass = np.array([g.pobj[t].mass for t in st["type"]], np.float64)
    weight = mass * gmag
    e_pp = rel_err(f["f_pp"], ref["f_pp"].astype(np.float64), weight)
    # walls and lifters keep the reference's arithmetic
    for key in ("f_wall", "t_wall", "f_lift", "t_lift"):
        np.testing.assert_array_equal(f[key], ref[key], err_msg=key)
    dt = float(np.float32(g.sim_info.InitalDelta_t))
    vel_scale = np.maximum(np.linalg.norm(ref["vel"], axis=1), gmag * dt)
    e_v = float((np.linalg.norm(st["vel"].astype(np.float64) - ref["vel"], axis=1) / vel_scale).max())
    print("%s: contracted law, step 1: force %.2e, velocity %.2e (relative, per particle)"
          % (name, e_pp, e_v))
    s.close()
    assert e_pp < TOL, e_pp
    assert e_v < TOL, e_v


def contact_force_scale(P, st):
    """Per particle (pid order) the largest force term of its sphere
    contacts, in FP64: the normal spring and dashpot (penetration plus the
    reference's 1e-5 cm), or the tangential tan_pre |v| / |v_rel| with |v|
    the contact-point speeds that v_t is formed from (the term whose
    rounding the law's tangential force carries); and the contact count."""
    from scipy.spatial import cKDTree
    rad = np.array([P.pobj[t].radius for t in range(P.n_p)], np.float64)[st["type"]]
    pos = st["pos"].astype(np.float64)
    pairs = np.array(sorted(cKDTree(pos).query_pairs(2.0 * rad.max())))
    dist = np.linalg.norm(pos[pairs[:, 0]] - pos[pairs[:, 1]], axis=1)
    # contacts as the FP32 test may count them (a hair beyond touching)
    touch = dist < (rad[pairs[:, 0]] + rad[pairs[:, 1]]) * (1.0 + 1e-6)
    contacts = int(touch.sum())
    # largest contact force per particle (normal spring-dashpot or the
    # reference's tangential force, tan_pre |v_t| / |v_rel|, in FP64), in pid order
    pp = [[P.pobj[a].PP[b] for b in range(P.n_p)] for a in range(P.n_p)]
    tp = st["type"].astype(np.int64)
    cp = pairs[touch]
    ta, tb = tp[cp[:, 0]], tp[cp[:, 1]]
    kn = np.array([pp[a][b].Kn for a, b in zip(ta, tb)])
    cn = np.array([pp[a][b].Cn for a, b in zip(ta, tb)])
    muk = np.array([pp[a][b].Fric_kinetic for a, b in zip(ta, tb)])
    m_all = np.array([P.pobj[t].mass for t in range(P.n_p)], np.float64)
    dt = float(np.float32(P.sim_info.InitalDelta_t))
    nrm = (pos[cp[:, 0]] - pos[cp[:, 1]]) / dist[touch][:, None]
    vel, avel = st["vel"].astype(np.float64), st["avel"].astype(np.float64)
    rvel = vel[cp[:, 0]] - vel[cp[:, 1]]
    vcpa = vel[cp[:, 0]] + np.cross(avel[cp[:, 0]], -nrm * rad[cp[:, 0]][:, None])
    vcpb = vel[cp[:, 1]] + np.cross(avel[cp[:, 1]], nrm * rad[cp[:, 1]][:, None])
    dv = vcpa - vcpb
    vt = dv - (dv * nrm).sum(1)[:, None] * nrm
    vr = np.linalg.norm(rvel, axis=1)
    tan_pre = 0.5 * (m_all[ta] + m_all[tb]) / dt * 0.05 * muk
    # the tangential force is tan_pre |v_t| / |v_rel| along v_t; v_t is formed
    # from the contact-point velocities, so its rounding scales with theirs
    f_t = tan_pre * (np.linalg.norm(vt, axis=1) + np.linalg.norm(vcpa, axis=1) +
                     np.linalg.norm(vcpb, axis=1)) / np.where(vr > 0, vr, 1.0)
    pen = np.abs(dist[touch] - (rad[cp[:, 0]] + rad[cp[:, 1]])) + 1e-5   # the reference's penetration
    f_n = np.abs(kn * pen) + np.abs(cn * (rvel * nrm).sum(1))
    fc = np.maximum(f_n, f_t)
    fmax = np.zeros(len(pos))
    np.maximum.at(fmax, cp[:, 0], fc)
    np.maximum.at(fmax, cp[:, 1], fc)
    fmax = fmax[np.argsort(st["pid"])]
    return fmax, contacts


def test_fast_law_vs_fp64_settled_silo(tmp_path):
    """20,000 spheres (r in [0.2, 0.4] cm) of the silo workload settled for
    20,000 steps with the hatch closed: a bed in contact, its overlaps set
    by the weight above.  One step's particle-particle forces, contracted
    and bit-exact, against the FP64 restatement of the reference law from
    that state.  Deep in a bed a particle's contact forces are many times
    its net force and its weight, and each carries its own rounding, so the
    scale of a particle here is the largest of its net force, its weight
    and the largest force term of its contacts (contact_force_scale: the
    reference's tangential force is formed from contact-point velocities
    that may be far larger than the slow relative motion it divides by).
    The reference's own FP32 arithmetic is printed beside it: against FP64
    it is off by more than its own force on the worst particle."""
    P, st0 = synth.silo_project(str(tmp_path), n=20000)
    s = device.Simulation(P, skin=0.1, use_graph=1)
    s.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"])
    s.step(20000)
    st = s.state()
    s.close()
    assert st["status"] == 0, device.decode_status(st["status"])
    fmax, contacts = contact_force_scale(P, st)
    assert 2 * contacts / len(st["pos"]) > 2.0, 2 * contacts / len(st["pos"])
    out = {}
    for fast in (0, 1):
        g = device.Simulation(P, capture_forces=1, fast_law=fast)
        g.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
        g.step(1)
        f = g.forces()["f_pp"]
        pid = g.state()["pid"]
        g.close()
        out[fast] = f[np.argsort(pid)]
    o = Restated("f64").init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d)
    o.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    o.step(1)
    f64 = o.forces()["f_pp"][np.argsort(o.state()["pid"])]
    mass = np.array([P.pobj[t].mass for t in range(P.n_p)], np.float64)
    weight = np.maximum(mass[st["type"][np.argsort(st["pid"])]] * 981.0, fmax)
    e_exact = rel_err(out[0], f64, weight)
    e_fast = rel_err(out[1], f64, weight)
    e_pair = rel_err(out[1], out[0].astype(np.float64), weight)
    print("settled silo, 20,000 spheres, %.1f contacts per particle: vs FP64 bit-exact %.2e "
          "contracted %.2e; contracted vs bit-exact %.2e"
          % (2 * contacts / len(st["pos"]), e_exact, e_fast, e_pair))
    assert e_pair < TOL, e_pair
