"""BxDF sampler checks on the oracle (CPU): where the library combines a BxDF's sampler with the guide by
one-sample MIS, the sampler must draw exactly the density its pdf reports.  Two checks per outgoing
direction: the pdf integrates to the probability that a sample is accepted (quadrature over the
sphere), and the sample mean of a smooth test function h(wi) / pdf(wi) over accepted samples matches
its integral over the pdf's support.  The conductor (visible-normal sampling) and the Lambert and
Oren-Nayar lobes pass; the reference's Plastic microfacet lobe reports a pdf without D(wh)
(Classic/Kernel.cpp:405-412) and is kept out of guiding, which the last test documents."""
import numpy as np
import pytest

from piper2_b200 import scenes


def _fib_sphere(m):
    i = np.arange(m) + 0.5
    z = 1 - 2 * i / m
    phi = np.pi * (1 + 5 ** 0.5) * i
    r = np.sqrt(1 - z * z)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1).astype(np.float32)


def _scene(materials):
    sd = scenes.SceneData(materials=materials)
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    sd.meshes = [scenes.MeshData(v, np.array([[0, 1, 2]], np.uint32), 0)]
    return sd


def _wo(theta):
    return np.array([np.sin(theta), 0.0, np.cos(theta)], np.float32)


def _check_sampler(osc, mat, theta, n=400_000, m=2_000_000, tol=0.01):
    wo = _wo(theta)
    rng = np.random.default_rng(int(theta * 1000) + mat)
    u = rng.uniform(0, 1, (n, 2)).astype(np.float32)
    wi, f, pdf = osc.bsdf_sample(mat, wo, u)
    ok = pdf > 0
    dirs = _fib_sphere(m)
    _, qpdf = osc.bsdf_eval(mat, wo, dirs)
    # the pdf integrates to the acceptance probability
    mass = qpdf.astype(np.float64).mean() * 4 * np.pi
    assert abs(mass - ok.mean()) <= tol, (mass, ok.mean())
    # E[h / pdf] over accepted samples = integral of h over the pdf's support
    h = lambda w: (1.0 + w[:, 0]) * (1.5 + w[:, 1]) * np.abs(w[:, 2])
    est = np.sum(h(wi[ok].astype(np.float64)) / pdf[ok]) / n
    exact = np.mean(h(dirs.astype(np.float64)) * (qpdf > 0)) * 4 * np.pi
    assert abs(est / exact - 1.0) <= tol, (est, exact)


@pytest.mark.parametrize("theta", [0.1, 0.7, 1.3])
@pytest.mark.parametrize("alpha", [0.1, 0.3, 0.6])
def test_conductor_sampler_density_matches_pdf(oracle, theta, alpha):
    sd = _scene([scenes.material("Conductor", color1=(0.9, 0.8, 0.7, 1.0), roughness=(alpha, alpha))])
    osc = oracle.OracleScene(sd, use_bvh=False)
    _check_sampler(osc, 0, theta, tol=0.02 if alpha == 0.1 else 0.01)


@pytest.mark.parametrize("theta", [0.2, 1.2])
@pytest.mark.parametrize("rough", [0.0, 0.5])
def test_matte_sampler_density_matches_pdf(oracle, theta, rough):
    sd = _scene([scenes.material("Matte", (0.7, 0.6, 0.5, 1.0), roughness=(rough, 0.0))])
    osc = oracle.OracleScene(sd, use_bvh=False)
    _check_sampler(osc, 0, theta)


def test_reference_plastic_pdf_is_not_its_sampler_density(oracle):
    """Plastic's glossy lobe (the reference's MicrofacetReflection) reports 1/4 / (wo.z p1 (p1 + p2)): its
    quadrature over the sphere is far from the acceptance probability.  Plain rendering keeps it for
    parity; guided rendering does not mix it with the guide."""
    sd = _scene([scenes.material("Plastic", (0.0, 0.0, 0.0, 1.0), (0.9, 0.9, 0.9, 1.0), roughness=(0.05, 0.0))])
    osc = oracle.OracleScene(sd, use_bvh=False)
    wo = _wo(0.5)
    _, qpdf = osc.bsdf_eval(0, wo, _fib_sphere(1_000_000))
    mass = qpdf.astype(np.float64).mean() * 4 * np.pi
    assert mass > 1.5 or mass < 0.5, mass
