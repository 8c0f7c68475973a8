"""Solver types and parameter structs of the reference's API.

    class ct(ct_params_default_t):      # compile-time parameters (opts.hpp:81-100)
        real_t = np.float64; n_dims = 2; n_eqns = 1; opts = opts.fct
    p = mpdata.rt_params_t(); p.grid_size = [101, 101]; p.n_iters = 2
    slv = mpdata(ct)                    # solvers::mpdata<ct_params_t> (solvers/mpdata.hpp:24-54)
"""
import numpy as np

from . import opts as _o


class ct_params_default_t:
    """Defaults of libmpdata++/opts.hpp:81-100."""
    real_t = np.float64
    n_dims = 1
    n_eqns = 1
    opts = _o.iga | _o.fct
    hint_norhs = 0
    delayed_step = 0
    var_dt = False
    prs_k_iters = 4
    prs_khn = False
    sgs_scheme = 0
    impl_tht = False
    vip_vab = 0       # noab (mpdata_rhs_vip_common.hpp:16-21)
    sptl_intrp = 0    # exact (formulae_mpdata_common.hpp:21-26): div_3rd spatial terms


class _rt_base:
    def __init__(self, **kw):
        self.grid_size = []
        self.dt = 0.0
        self.di = self.dj = self.dk = 0.0
        self.max_abs_div_eps = None   # default: machine epsilon of real_t (solver_common.hpp:220)
        self.max_courant = 0.5
        self.n_iters = 2              # mpdata_common.hpp:77
        self.upwind_filter_freq = 0
        for k, v in kw.items():
            setattr(self, k, v)


class mpdata:
    """solvers::mpdata<ct_params_t>: oscillatory or FCT variant selected by opts::fct."""

    class rt_params_t(_rt_base):
        pass

    def __init__(self, ct):
        self.ct = ct
        if ct.var_dt:
            raise NotImplementedError("var_dt is not built on this backend")


# right-hand-side schemes (mpdata_rhs.hpp:19-25), pressure schemes (mpdata_rhs_vip_prs.hpp:17-30)
# and velocity absorbers (mpdata_rhs_vip_common.hpp:16-21)
euler_a, euler_b, trapez, mixed = range(4)
mr, cr, pc, gcrk = range(4)
noab, expl, impl = range(3)


class boussinesq:
    """solvers::boussinesq<ct_params_t> (solvers/boussinesq.hpp:20-52): explicit
    buoyancy (boussinesq_expl.hpp) or, with ct.impl_tht, the implicit theta
    perturbation form (boussinesq_impl.hpp); trapezoidal rhs coupling, GCR
    pressure solve, velocity absorber ct.vip_vab (noab, expl or impl).  The
    absorber coefficient and relaxed states are the scalar arrays "vab_coeff"
    and "vab_relax0..2" (vab_coefficient(), vab_relaxed_state(d))."""

    class rt_params_t(_rt_base):
        def __init__(self, **kw):
            self.prs_tol = 1e-7
            self.g = 9.81
            self.Tht_ref = 0.0
            self.precond = "identity"   # or "learned"
            self.prs_fp64 = False
            super().__init__(**kw)

    def __init__(self, ct):
        self.ct = ct
        if getattr(ct, "rhs_scheme", trapez) != trapez:
            raise NotImplementedError("only the trapez rhs scheme is built")
        if getattr(ct, "prs_scheme", cr) not in (cr, gcrk):
            raise NotImplementedError("only the cr / gcrk pressure schemes are built")

    def fill_config(self, cfg, p):
        from . import _lib
        ct = self.ct
        ix = ct.ix
        cfg.prs_scheme = _lib.PRS_CR if getattr(ct, "prs_scheme", cr) == cr else _lib.PRS_GCRK
        cfg.prs_k_iters = int(getattr(ct, "prs_k_iters", 4))
        cfg.prs_tol = float(p.prs_tol)
        cfg.g = float(p.g)
        cfg.tht_ref = float(p.Tht_ref)
        cfg.ix_u = int(ix.vip_i)
        cfg.ix_v = int(ix.vip_j) if int(ct.n_dims) == 3 else -1
        cfg.ix_w = int(ix.vip_k if int(ct.n_dims) == 3 else ix.vip_j)
        cfg.ix_tht = int(ix.tht)
        cfg.precond = _lib.PRECOND_LEARNED if p.precond == "learned" else _lib.PRECOND_IDENTITY
        cfg.prs_fp64 = 1 if p.prs_fp64 else 0
        cfg.impl_tht = 1 if getattr(ct, "impl_tht", False) else 0
        cfg.vip_vab = int(getattr(ct, "vip_vab", noab))
