"""Generate golden vectors from the reference's own CUDA kernels.

Runs on a GPU box with ``oracle/_ref/libglide_ref.so`` (built from the
reference tree by ``oracle/build_ref.py``).  Inputs are the seeded 32x32
dome case (plus random velocities / tangents for the single-operator
cases); outputs are the reference kernels' FP32 results.  Writes
``tests/golden/reference_kernels_32.npz``, which ``tests/test_golden.py``
uses to pin the FP64 NumPy oracle.

Usage:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def main(out=os.path.join(ROOT, "tests", "golden", "reference_kernels_32.npz")):
    import torch
    from conftest import random_state
    from glide_b200.synthetic import dome_case
    from oracle import ref_replay as R

    st = random_state(n=32, seed=0)
    f32 = {k: (v.astype(np.float32) if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    res = {f"in_{k}": v for k, v in f32.items() if isinstance(v, np.ndarray)}
    res["dx"] = np.float32(st["dx"])
    res["dt"] = np.float32(st["dt"])
    T = lambda a: torch.as_tensor(a, device="cuda")

    def grid(gl=False):
        g = R.RefGrid(32, 32, st["dx"], st["dt"], gl_derivatives=gl)
        for k in ("u", "v", "H", "bed", "B", "beta", "mask", "gamma", "f_u", "f_v", "f_H", "d_u", "d_v", "d_H"):
            getattr(g, k).copy_(T(f32[k]))
        return g

    g = grid()
    g.compute_residual()
    res.update(out_r_u=g.r_u.cpu().numpy(), out_r_v=g.r_v.cpu().numpy(), out_r_H=g.r_H.cpu().numpy())
    for gl in (False, True):
        g = grid(gl)
        g.compute_jvp()
        res.update({f"out_jvp{int(gl)}_u": g.j_u.cpu().numpy(), f"out_jvp{int(gl)}_v": g.j_v.cpu().numpy(),
                    f"out_jvp{int(gl)}_H": g.j_H.cpu().numpy()})
        g.lambda_u.copy_(T(f32["f_u"]))
        g.lambda_v.copy_(T(f32["f_v"]))
        g.lambda_H.copy_(T(f32["f_H"]))
        g.compute_vjp()
        res.update({f"out_vjp{int(gl)}_u": g.l_u.cpu().numpy(), f"out_vjp{int(gl)}_v": g.l_v.cpu().numpy(),
                    f"out_vjp{int(gl)}_H": g.l_H.cpu().numpy()})
    g = grid()
    g.lambda_u.copy_(T(f32["d_u"]))
    g.lambda_v.copy_(T(f32["d_v"]))
    res["out_grad_beta"] = g.compute_grad_beta().cpu().numpy()

    # one Vanka sweep (velocities scaled down so the local Newton is well posed)
    g = grid()
    g.u.mul_(0.02)
    g.v.mul_(0.02)
    res["in_vanka_u"], res["in_vanka_v"] = g.u.cpu().numpy(), g.v.cpu().numpy()
    g.vanka_sweep(1)
    res.update(out_vanka_u=g.u.cpu().numpy(), out_vanka_v=g.v.cpu().numpy(), out_vanka_H=g.H.cpu().numpy())
    # one local sweep with a hand-set error mask
    g = grid()
    g.u.copy_(T(res["in_vanka_u"]))
    g.v.copy_(T(res["in_vanka_v"]))
    em = np.zeros((32, 32), np.float32)
    em[3, 20] = 1
    em[27, 13] = 1
    res["in_error_mask"] = em
    g.error_mask.copy_(T(em))
    g.vanka_sweep_local(1)
    res.update(out_vlocal_u=g.u.cpu().numpy(), out_vlocal_v=g.v.cpu().numpy(), out_vlocal_H=g.H.cpu().numpy())
    # one adjoint colour pair from lambda = d
    g = grid()
    for k, s in (("lambda_u", "d_u"), ("lambda_v", "d_v"), ("lambda_H", "d_H"), ("f_adj_u", "f_u"),
                 ("f_adj_v", "f_v"), ("f_adj_H", "f_H")):
        getattr(g, k).copy_(T(f32[s]))
    g.vanka_sweep_adjoint(1, omega=1.0)
    res.update(out_vadj_u=g.lambda_u.cpu().numpy(), out_vadj_v=g.lambda_v.cpu().numpy(),
               out_vadj_H=g.lambda_H.cpu().numpy())
    # transfers
    rng = np.random.default_rng(9)
    uf, vf, hf = (rng.standard_normal(s).astype(np.float32) for s in ((16, 25), (17, 24), (16, 24)))
    uc, vc, hc = (rng.standard_normal(s).astype(np.float32) for s in ((8, 13), (9, 12), (8, 12)))
    res.update(tr_uf=uf, tr_vf=vf, tr_hf=hf, tr_uc=uc, tr_vc=vc, tr_hc=hc)
    E = lambda s: torch.empty(s, dtype=torch.float32, device="cuda")
    res["tr_restrict_u"] = R.restrict_vfacet(T(uf), E((8, 13))).cpu().numpy()
    res["tr_restrict_v"] = R.restrict_hfacet(T(vf), E((9, 12))).cpu().numpy()
    res["tr_restrict_c"] = R.restrict_cell_centered(T(hf), E((8, 12))).cpu().numpy()
    res["tr_restrict_max"] = R.restrict_max_pool(T(hf), E((8, 12))).cpu().numpy()
    res["tr_prolong_u_lin"] = R.prolongate_vfacet(T(uc), E((16, 25)), smooth=False).cpu().numpy()
    res["tr_prolong_u_bil"] = R.prolongate_vfacet(T(uc), E((16, 25)), smooth=True).cpu().numpy()
    res["tr_prolong_v_lin"] = R.prolongate_hfacet(T(vc), E((17, 24)), smooth=False).cpu().numpy()
    res["tr_prolong_v_bil"] = R.prolongate_hfacet(T(vc), E((17, 24)), smooth=True).cpu().numpy()
    res["tr_prolong_c_inj"] = R.prolongate_cell_centered(T(hc), E((16, 24)), smooth=False).cpu().numpy()
    res["tr_prolong_c_bil"] = R.prolongate_cell_centered(T(hc), E((16, 24)), smooth=True).cpu().numpy()

    # one forward step (1 V-cycle, 3 levels) and one adjoint V-cycle on the dome case
    c = dome_case(0, n=32, dx=10000.0, n_levels=3)
    ph = R.RefIcePhysics(32, 32, c.dx, n_levels=3, thklim=c.thklim)
    ph.set_geometry(c.bed, c.thickness)
    ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    u, v, H = ph.forward(c.dt, n_vcycles=1)
    res.update(step_u=u.cpu().numpy(), step_v=v.cpu().numpy(), step_H=H.cpu().numpy())
    rng = np.random.default_rng(3)
    dLu = (rng.standard_normal((32, 33)) * 1e-3).astype(np.float32)
    dLv = (rng.standard_normal((33, 32)) * 1e-3).astype(np.float32)
    gb = ph.adjoint(dLu, dLv, np.zeros((32, 32), np.float32), n_vcycles=1)
    res.update(step_dLu=dLu, step_dLv=dLv, step_grad_beta=gb.cpu().numpy())
    np.savez_compressed(out, **res)
    print("wrote", out, sum(v.nbytes for v in res.values() if isinstance(v, np.ndarray)), "bytes")


if __name__ == "__main__":
    main()
