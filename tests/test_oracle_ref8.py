"""The oracle's 8-rank form (REF8) of Force (no GPU needed).

The reference runs on exactly eight MPI ranks, one per coordinate octant
(mpienv.f90:19, main.f90:840-862).  Each rank walks its own trees, then the
pruned trees of the other seven (CopyTree, tree.f90:1167-1777;
RebuildGhostTree, 1781-1853; Ghost_Tree_*, 1856-2330), where a twig that the
sender did not expand arrives as a bare monopole leaf.  REF8 restates that in
one process; it is not a device gate, it measures how far the real 8-rank
reference sits from the single-domain form (REF1) the device path matches.

Pins that do not come from REF8 itself:
  * one populated octant: REF8 is REF1 bit for bit (no ghosts);
  * theta -> 0: every twig is expanded and opened, REF8 is the direct sum;
  * a far cluster: the receiver sees one point charge qeff at the charge
    centre with the leaf law, computed here by hand;
  * the contact case of every pair of octants, from the octant coordinates.
"""
import math

import numpy as np
import pytest

import oracle
from tree_b200 import cloud, units

EPS = units.EPS


def _params(theta=0.5, physics=oracle.PHYS_REF, rs=0.003):
    lam = units.kelbg_lambdas(50.0)
    return oracle.make_params(theta=theta, rs=rs, dx_ei=0.01, dx_ii=0.1,
                              lambdas=lam, physics=physics)


def _rel(f, g):
    n = np.linalg.norm(g, axis=1)
    return np.linalg.norm(f - g, axis=1) / np.maximum(n, 1e-3 * n.max())


@pytest.mark.parametrize("physics", [oracle.PHYS_REF, oracle.PHYS_KELBG])
def test_one_octant_is_the_single_domain_form(oracle_lib, physics):
    rng = np.random.default_rng(3)
    xi = np.abs(rng.standard_normal((700, 3))) * 20 + 0.5
    xe = np.abs(xi + rng.standard_normal(xi.shape) * 0.3) + 0.1
    p = _params(physics=physics)
    r1 = oracle.force(xe, xi, p)
    r8 = oracle.force_ref8(xe, xi, p)
    assert r8["ref8"]["n_el"][7] == 700 and r8["ref8"]["n_ion"][7] == 700
    assert r8["ref8"]["n_m2p_ghost"] == 0 and r8["ref8"]["n_p2p_ghost"] == 0
    np.testing.assert_array_equal(r8["f_el"], r1["f_el"])
    np.testing.assert_array_equal(r8["f_ion"], r1["f_ion"])
    np.testing.assert_array_equal(r8["rdf_ei"], r1["rdf_ei"])
    np.testing.assert_array_equal(r8["rdf_ii"], r1["rdf_ii"])
    # (energies are OpenMP reductions, combined in the threads' finishing order)
    assert r8["epot_e"] == pytest.approx(r1["epot_e"], rel=1e-12)
    assert r8["epot_i"] == pytest.approx(r1["epot_i"], rel=1e-12)


@pytest.mark.parametrize("physics", [oracle.PHYS_REF, oracle.PHYS_KELBG])
def test_theta_zero_is_the_direct_sum(oracle_lib, physics):
    rng = np.random.default_rng(4)
    xi = rng.standard_normal((300, 3)) * 30
    xe = xi + rng.standard_normal(xi.shape) * 2.0
    p = _params(theta=1e-12, physics=physics)
    r8 = oracle.force_ref8(xe, xi, p)
    d = oracle.direct(xe, xi, p)
    r1 = oracle.force(xe, xi, p)
    f8 = np.vstack([r8["f_el"], r8["f_ion"]])
    assert _rel(f8, np.vstack([d["f_el"], d["f_ion"]])).max() <= 1e-12
    assert r8["epot_e"] + r8["epot_i"] == pytest.approx(d["epot"], rel=1e-12)
    # every pair is a leaf pair in both forms: the same RDF counts
    np.testing.assert_array_equal(r8["rdf_ei"], r1["rdf_ei"])
    np.testing.assert_array_equal(r8["rdf_ii"], r1["rdf_ii"])
    assert r8["stats"]["n_m2p"] == 0


def test_unexpanded_twig_arrives_as_a_point_charge(oracle_lib):
    """Five ions 0.01 um apart near (5, 5, 5) (octant 7) and one electron at
    (-3, 5, 5) (octant 6, across the y-z face): the ion tree's root is far
    from the plane x = 0 (lx/theta + dx << 5), so rank 7 sends it without
    children and the electron feels one charge +5 at the ions' charge centre
    through the e-i leaf law (tree.f90:2202-2216)."""
    xi = np.array([[5.0, 5.0, 5.0], [5.01, 5.0, 5.0], [5.0, 5.01, 5.0],
                   [5.0, 5.0, 5.01], [5.01, 5.01, 5.01]])
    xe = np.array([[-3.0, 5.0, 5.0]])
    rs = 0.003
    r8 = oracle.force_ref8(xe, xi, _params(theta=0.5, rs=rs))
    assert r8["ref8"]["ghost_nodes_i"] == 7  # the lone root, once per other rank
    cc = xi.mean(axis=0)  # equal charges: the charge centre is the mean
    d = xe[0] - cc
    r = float(np.linalg.norm(d))
    ff = -1.0 * EPS * 5.0
    e = math.exp(-r / rs)
    want = ff * d * (1.0 / r - e * (1.0 / r + 1.0 / rs)) / r**2
    np.testing.assert_allclose(r8["f_el"][0], want, rtol=1e-12)
    # the single-domain form sees the cluster through its multipole instead
    r1 = oracle.force(xe, xi, _params(theta=0.5, rs=rs))
    assert not np.array_equal(r1["f_el"][0], r8["f_el"][0])
    assert np.linalg.norm(r1["f_el"][0] - want) <= 1e-4 * np.linalg.norm(want)


def test_contact_cases_from_octant_coordinates(oracle_lib):
    """CriterionFind (main.f90:865-925) through the oracle: a pair of particles
    in octants a and b whose ghost trees are pruned by the case's distance.
    Each case is checked by the pruning it causes: a lone twig at distance
    d from the contact set is expanded exactly when s/theta + dx > d."""
    # octant index = 4 z + 2 y + x bits (id_FINDER); the contact set of two
    # octants is spanned by the axes on which they agree
    def case(a, b):
        same = [((a >> k) & 1) == ((b >> k) & 1) for k in range(3)]
        table = {(False, True, True): 1, (True, False, True): 2, (True, True, False): 3,
                 (True, False, False): 4, (False, True, False): 5,
                 (False, False, True): 6, (False, False, False): 7}
        return table[tuple(same)]

    def dist(c, x):
        axes = {1: [0], 2: [1], 3: [2], 4: [1, 2], 5: [0, 2], 6: [0, 1], 7: [0, 1, 2]}[c]
        return math.sqrt(sum(x[k] ** 2 for k in axes))

    centre = np.array([2.0, 3.0, 4.0])
    for b in range(8):
        sgn = np.array([1 if (b >> k) & 1 else -1 for k in range(3)], float)
        # two ions 0.2 apart in octant b; one electron in every other octant
        xi = np.vstack([centre * sgn, centre * sgn + 0.2 * sgn])
        xe = np.array([[(1 if (a >> k) & 1 else -1) * 7.0 for k in range(3)]
                       for a in range(8) if a != b])
        for theta in (0.02, 0.5):
            r8 = oracle.force_ref8(xe, xi, _params(theta=theta))
            # the ion root (a twig of 2) is expanded into 2 leaves (3 nodes) or
            # sent alone (1 node) on each of the 7 links
            expanded = 0
            s = 0.2 / 1.0  # MAXVAL(lx) of the 2-ion root box
            cc = (xi[0] + xi[1]) / 2
            dx = float(np.linalg.norm(cc - (xi[0] + xi[1]) / 2))
            for a in range(8):
                if a == b:
                    continue
                if s / theta + dx > dist(case(a, b), cc):
                    expanded += 1
            assert r8["ref8"]["ghost_nodes_i"] == 3 * expanded + (7 - expanded)


def test_plain_method_4096_ref8_against_ref1(oracle_lib):
    """The 4,096-particle plain-method cloud two steps in (electrons 0.3 um
    off their ions): how far the 8-rank reference is from the single-domain
    form, against the FP64 direct sum.  Both forms carry errors of the same
    order at theta = 0.5; their difference is of that order, not smaller."""
    c = cloud.make_cloud(4096, seed=101)
    rng = np.random.Generator(np.random.Philox(102))
    xe = c.x_ion + rng.standard_normal(c.x_ion.shape) * 0.3
    xi = c.x_ion
    lam = units.kelbg_lambdas(50.0)
    p = oracle.make_params(theta=0.5, rs=lam[1], dx_ei=0.01, dx_ii=0.1, lambdas=lam,
                           physics=oracle.PHYS_REF)
    r1 = oracle.force(xe, xi, p)
    r8 = oracle.force_ref8(xe, xi, p)
    d = oracle.direct(xe, xi, oracle.make_params(theta=1e-12, rs=lam[1], lambdas=lam,
                                                 physics=oracle.PHYS_REF))
    f1 = np.vstack([r1["f_el"], r1["f_ion"]])
    f8 = np.vstack([r8["f_el"], r8["f_ion"]])
    fd = np.vstack([d["f_el"], d["f_ion"]])
    e81 = _rel(f8, f1)
    e1 = _rel(f1, fd)
    e8 = _rel(f8, fd)
    rms = lambda e: float(np.sqrt(np.mean(e ** 2)))  # noqa: E731
    print(f"REF8 vs REF1 rms {rms(e81):.2e} max {e81.max():.2e}; "
          f"REF1 vs direct rms {rms(e1):.2e}; REF8 vs direct rms {rms(e8):.2e}; "
          f"ghost nodes e/i {r8['ref8']['ghost_nodes_e']}/{r8['ref8']['ghost_nodes_i']}")
    assert sum(r8["ref8"]["n_el"]) == 2048 and min(r8["ref8"]["n_el"]) > 150
    assert 1e-6 < rms(e81) < 1e-3
    assert rms(e8) < 1e-3 and rms(e1) < 1e-3
    assert r8["epot_e"] == pytest.approx(r1["epot_e"], rel=1e-4)
