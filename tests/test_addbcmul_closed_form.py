"""CPU: the closed form the persistent GMRES cycle uses for memLS's two
ADDBCMUL passes on a Krylov product (flowsolver/src/memLS.f90:206-268).

memLS applies, to w = K u (u the previous basis vector):
  op 0 (ADD):  S0_f = valM_f . u,  then w += sum_f coef0_f S0_f valM_f
  op 1 (PRE):  S1_f = valM_f . w,  then w += sum_f coef1_f S1_f valM_f
with every face dot taken before any update of the same pass.  The kernel
forms S0_f and T_f = valM_f . (K u) in one sweep and uses
  S1_f = T_f + sum_g coef0_g S0_g (valM_f . valM_g)
so one pass over the rows applies both updates.  This checks the identity in
FP64 for faces that share nodes (outlets splitting one cap share rim nodes).
"""
import numpy as np


def _two_passes(w, u, faces, coef0, coef1):
    w = w.copy()
    s0 = [vf @ u for vf in faces]
    for c, s, vf in zip(coef0, s0, faces):
        w += c * s * vf
    s1 = [vf @ w for vf in faces]
    for c, s, vf in zip(coef1, s1, faces):
        w += c * s * vf
    return w


def _closed_form(w, u, faces, coef0, coef1):
    s0 = np.array([vf @ u for vf in faces])
    t = np.array([vf @ w for vf in faces])
    gram = np.array([[vf @ vg for vg in faces] for vf in faces])
    s1 = t + gram @ (np.asarray(coef0) * s0)
    out = w.copy()
    for f, vf in enumerate(faces):
        out += (coef0[f] * s0[f] + coef1[f] * s1[f]) * vf
    return out


def test_closed_form_matches_two_passes_with_shared_nodes():
    rng = np.random.default_rng(4)
    n = 3 * 500
    for nface in (1, 2, 3, 8):
        faces = []
        for f in range(nface):
            vf = np.zeros(n)
            nodes = rng.choice(n // 3, size=40, replace=False)
            if f > 0:   # share a few rim nodes with the previous face
                prev = np.nonzero(faces[-1])[0][::3][:5] // 3
                nodes = np.unique(np.concatenate([nodes, prev]))
            for a in nodes:
                vf[3 * a:3 * a + 3] = rng.standard_normal(3)
            faces.append(vf)
        res = rng.uniform(10.0, 200.0, nface)
        nS = np.array([vf @ vf for vf in faces])
        coef0 = res
        coef1 = -res / (1.0 + res * nS)
        w = rng.standard_normal(n)
        u = rng.standard_normal(n)
        ref = _two_passes(w, u, faces, coef0, coef1)
        got = _closed_form(w, u, faces, coef0, coef1)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), nface
