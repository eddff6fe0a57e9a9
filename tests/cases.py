"""Shared parity cases: the same parameters drive the CPU restatement and the engine."""

DENDRITE_REF = dict(dt=5e-5, dx=0.02, delta=0.5, tau=0.0003, epsilon=0.01, alpha=0.9, gamma=40.0, Delta=0.25,
                    metric_p=0.01, metric_T=1e-5)
MODELB_REF = dict(dt=0.001, dx=1.0, chi_xy=0.0, chi_xz=0.0, chi_yz=0.0, chi_xb=0.0, chi_yb=0.0, chi_zb=4.0,
                  vx=1, vy=1, vz=2, rx=1, ry=1, rz=2, n=1, m=1, eps_x=4.0, eps_y=4.0, eps_z=4.0, eps_phi=0.01,
                  M_x=1.0, M_y=1.0, M_z=1.0, M_phi=1.0, x0=0.2, y0=0.2, z0=0.01, K=100.0, z_crit=0.4, p_gel=1.0,
                  k_0=1.0, metric_eps=1e-6)
KH_REF = dict(dt=0.0002, dx=0.002, dy=0.002, metric_eps=0.0, gamma=5.0 / 3.0)

# oracle key -> engine Config field
_MB_MAP = {"M_x": "mob_x", "M_y": "mob_y", "M_z": "mob_z", "M_phi": "mob_phi"}


def dendrite_cfg(prm, nx, ny, nz, block, precision=0, bc=0, **kw):
    import dba_b200
    c = dba_b200.config("dendrite", nx=nx, ny=ny, nz=nz, block=block, precision=precision, bc=bc)
    for k in ("dt", "dx", "delta", "tau", "epsilon", "alpha", "gamma", "Delta", "metric_p", "metric_T"):
        setattr(c, k, prm[k])
    c.dy = c.dz = prm["dx"]
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def modelb_cfg(prm, nx, ny, nz, block, precision=0, conserved=0, **kw):
    import dba_b200
    c = dba_b200.config("modelb", nx=nx, ny=ny, nz=nz, block=block, precision=precision, conserved=conserved)
    for k, v in prm.items():
        setattr(c, _MB_MAP.get(k, k), v)
    c.dy = c.dz = prm["dx"]
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def kh_cfg(prm, nx, ny, block, precision=0, conserved=0, **kw):
    import dba_b200
    c = dba_b200.config("kh", nx=nx, ny=ny, nz=1, block=block, precision=precision, conserved=conserved)
    c.dt, c.dx, c.dy, c.metric_eps, c.kh_gamma = prm["dt"], prm["dx"], prm["dy"], prm["metric_eps"], prm["gamma"]
    c.dz = prm["dx"]
    for k, v in kw.items():
        setattr(c, k, v)
    return c
