"""The ensemble's reference-law mode (BLAZE_LAW_REFERENCE) against oracle A
(the reference's own kernels compiled as host C++) system by system, on a
sample of the batched workload's systems.

The batched workload draws radii uniformly from [0.1, 0.2] cm; the
reference holds one radius per particle object (at most six objects per
world), so the sampled systems take their radii from six bins of that
range.  Their counts, friction and restitution are the batched workload's
(counts log-uniform in [2,000, 50,000], seed 3; mu in [0.2, 0.8],
restitution in [0.3, 0.9]).  The ensemble settles the sampled systems
together from their lattices; the state it reaches is then given to oracle
A, one system at a time, as the project synth.box_system_project writes
for the system (box of six quads, one particle object per radius), and both
take the same steps from there.

Bar: forces of the next step within 1e-5 of each particle's scale (the
larger of its net contact force and its weight) -- the contacts are summed
in list order here and in cell order there, and the masses and damping
coefficients are formed from the same expressions in another order of the
same double arithmetic, so agreement is to rounding, not bit for bit;
positions and velocities after 20 steps within 1e-5 relative.
"""
import tempfile

import numpy as np
import pytest

from bindings import RefHost, ref_available
from blaze import ensemble as E
from blaze import synth

pytestmark = pytest.mark.gpu

RHO = 2500.0
SAMPLE = 4
PREROLL = 2500
TOL = 1e-5


def sampled_systems():
    counts = synth.batched_counts(512, seed=3)
    rng = np.random.default_rng(3)
    mus = rng.uniform(0.2, 0.8, len(counts))
    rests = rng.uniform(0.3, 0.9, len(counts))
    # a seeded sample, kept to systems of at most 12,000 spheres so that
    # oracle A's steps stay short
    small = np.nonzero(counts <= 12000)[0]
    pick = np.sort(np.random.default_rng(21).choice(small, SAMPLE, replace=False))
    S, W, p, r = synth.box_ensemble(counts[pick], mus=mus[pick], restitutions=rests[pick],
                                    seed=3, rho=RHO)
    edges = np.linspace(0.1, 0.2, 7)
    centres = (0.5 * (edges[:-1] + edges[1:])).astype(np.float32)
    rb = centres[np.clip(np.digitize(r, edges) - 1, 0, 5)]
    return pick, S, W, p, rb


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_reference_law_systems_against_oracle_a():
    pick, S, W, p, r = sampled_systems()
    ens = E.Ensemble(S, W, law=E.LAW_REFERENCE, dt=1e-5, skin=0.02, use_graph=1,
                     capture_forces=1)
    ens.set_state(p, r)
    ens.step(PREROLL)
    st = ens.state()
    assert st["status"] == 0, st["status"]
    ens.step(1)
    f1, _ = ens.forces()
    s1 = ens.state()
    ens.step(19)
    s20 = ens.state()
    ens.close()
    off = np.concatenate([[0], np.cumsum([s.n for s in S])])
    for k, sys_id in enumerate(pick):
        m0 = st["sys"] == k
        pid = st["pid"][m0] - off[k]
        order = np.argsort(pid)
        L, H = -W[6 * k + 1].p[3], -W[6 * k + 5].p[3]
        with tempfile.TemporaryDirectory() as d:
            P, types = synth.box_system_project(d, "Sys%d" % sys_id, S[k], L, H,
                                                r[off[k]:off[k + 1]], RHO)
        R = RefHost().init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d, threads=8,
                           capture=True)
        pos = st["pos"][m0][order]
        R.set_state(pos, st["vel"][m0][order], st["avel"][m0][order], types,
                    np.arange(len(pos), dtype=np.int32))
        assert R.step(1) == 0
        fr = R.forces()
        ra = R.state()
        ia = np.argsort(ra["pid"])
        mass = np.array([P.pobj[t].mass for t in range(P.n_p)], np.float64)[types]
        g = np.array([S[k].gravity[q] for q in range(3)], np.float64)
        # oracle A's f_pp starts from the weight; the ensemble reports contacts only
        fa = (fr["f_pp"][ia].astype(np.float64) - mass[:, None] * g) + fr["f_wall"][ia]
        m1 = s1["sys"] == k
        fg = f1[m1][np.argsort(s1["pid"][m1] - off[k])].astype(np.float64)
        scale = np.maximum(np.linalg.norm(fa, axis=1), mass * np.linalg.norm(g))
        e_f = float((np.linalg.norm(fg - fa, axis=1) / scale).max())
        contacts = float((np.linalg.norm(fa, axis=1) > 0).mean())
        assert R.step(19) == 0
        rb_ = R.state()
        ib = np.argsort(rb_["pid"])
        m20 = s20["sys"] == k
        o20 = np.argsort(s20["pid"][m20] - off[k])
        e_x = float(np.abs(s20["pos"][m20][o20] - rb_["pos"][ib]).max() / max(L, H))
        vs = max(float(np.abs(rb_["vel"]).max()), 1e-30)
        e_v = float(np.abs(s20["vel"][m20][o20] - rb_["vel"][ib]).max() / vs)
        print("system %d (%d spheres, mu %.2f, e %.2f): %.0f %% in contact; step 1 force %.2e; "
              "after 20 steps position %.2e velocity %.2e"
              % (sys_id, S[k].n, S[k].mu, S[k].restitution, 100 * contacts, e_f, e_x, e_v))
        assert contacts > 0.5
        assert e_f < TOL, e_f
        assert e_x < TOL and e_v < TOL, (e_x, e_v)
