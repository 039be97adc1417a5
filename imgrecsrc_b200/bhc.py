"""Polychromatic beam-hardening model over torch tensors (include/ctprj.h,
ctprj_bhc_*), the GPU counterpart of bhc/Spline.m (b1Iout) with
bhc/poissLAlpha.m and bhc/poissLI.m.

Per ray i: s_i = Ts (A x)_i; BL_i = sum_j Ie_j b_j(s_i) over degree-1 B-spline
basis functions on J + 2 mass-attenuation nodes; the Poisson negative
log-likelihood f = sum_i BL_i - m_i - m_i log(BL_i / m_i) of the measured
intensity m (counts / I0), and its gradients in x (through Ts A^T) and in Ie.
Spline arithmetic and reductions are FP64 on the GPU.
"""
import ctypes

import numpy as np

from ._lib import LoopOpts, LoopStats, check, lib
from .projector import _dev_ptr, _stream_handle


def kappa_nodes(J, kmin=1e-2, kmax=1e2):
    """J log-spaced values on [kmin, kmax] padded with one node on each side at
    the grid's ratio (the node rule of bhc/beamhardenSpline.m:164-165)."""
    kappa = np.logspace(np.log10(kmin), np.log10(kmax), J)
    q = kappa[1] / kappa[0]
    return np.concatenate([[kappa[0] / q], kappa, [kappa[-1] * q]])


def _dptr(t, n, dtype):
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise TypeError("expected a contiguous CUDA %s tensor" % dtype)
    if t.numel() != n:
        raise ValueError("expected %d elements, got %d" % (n, t.numel()))
    return ctypes.c_void_p(t.data_ptr())


class BHCModel:
    """Fused forward (projection + per-ray spline epilogue) and hand-written
    adjoint on one Projector's geometry."""

    def __init__(self, projector, nodes, Ts):
        self.projector = projector
        self.nodes = np.ascontiguousarray(nodes, np.float64)
        self.J = self.nodes.size - 2
        self.Ts = float(Ts)
        self._m = ctypes.c_void_p()
        check(lib().ctprj_bhc_create(projector._plan, self.J, self.nodes.ctypes.data,
                                     self.Ts, ctypes.byref(self._m)))
        g = projector.geometry
        self.nrays = g.np * g.prjWidth
        self.noise = "poisson"

    def close(self):
        if self._m:
            lib().ctprj_bhc_destroy(self._m)
            self._m = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _args(self, x, Ie, imea):
        import torch
        pr = self.projector
        return (_dev_ptr(x, pr.img_shape, pr.device) if x is not None else None,
                _dptr(Ie, self.J, torch.float64) if Ie is not None else None,
                _dptr(imea, self.nrays, torch.float32) if imea is not None else None)

    def forward(self, x, Ie, imea, save=True, out=None, stream=None):
        """f (a 1-element float64 CUDA tensor) for density x (n, n), spectrum
        coefficients Ie (J, float64) and measured intensity imea (np, prjWidth)."""
        import torch
        out = torch.empty(1, dtype=torch.float64, device=x.device) if out is None else out
        px, pI, pm = self._args(x, Ie, imea)
        check(lib().ctprj_bhc_forward(self._m, px, pI, pm, _dptr(out, 1, torch.float64),
                                      1 if save else 0, _stream_handle(stream, self.projector.device)))
        return out

    def terms(self, sino, Ie, imea, save=True, out=None, stream=None):
        """The same likelihood from a plain sinogram (unfused path)."""
        import torch
        out = torch.empty(1, dtype=torch.float64, device=sino.device) if out is None else out
        pr = self.projector
        _, pI, pm = self._args(None, Ie, imea)
        check(lib().ctprj_bhc_terms(self._m, _dev_ptr(sino, pr.sino_shape, pr.device), pI, pm,
                                    _dptr(out, 1, torch.float64), 1 if save else 0,
                                    _stream_handle(stream, pr.device)))
        return out

    def basis(self, sino, out=None, stream=None):
        """The (rays, J) FP64 basis matrix b_j(Ts * sino_i)."""
        import torch
        pr = self.projector
        out = torch.empty(self.nrays, self.J, dtype=torch.float64, device=sino.device) if out is None else out
        check(lib().ctprj_bhc_basis(self._m, _dev_ptr(sino, pr.sino_shape, pr.device),
                                    _dptr(out, self.nrays * self.J, torch.float64),
                                    _stream_handle(stream, pr.device)))
        return out

    def set_noise(self, noise):
        """'poisson' (bhc/poissLAlpha.m, the default) or 'gaussian'
        (bhc/gaussLAlpha.m: log-domain least squares)."""
        code = {"poisson": 0, "gaussian": 1}[noise]
        check(lib().ctprj_bhc_set_noise(self._m, code))
        self.noise = noise

    def hessian(self, v, Ie, imea, Hv=True, vHv=True, stream=None):
        """Density Hessian at the saved forward state applied to v:
        (Ts A^T (h * Ts A v) as (n, n) float32 or None, v'Hv as a float or None)."""
        import torch
        pr = self.projector
        hv = torch.empty(pr.img_shape, dtype=torch.float32, device=v.device) if Hv else None
        q = torch.zeros(1, dtype=torch.float64, device=v.device) if vHv else None
        check(lib().ctprj_bhc_hessian(self._m, _dptr(Ie, self.J, torch.float64),
                                      _dptr(imea, self.nrays, torch.float32),
                                      _dev_ptr(v, pr.img_shape, pr.device),
                                      None if hv is None else _dev_ptr(hv, pr.img_shape, pr.device),
                                      None if q is None else q.data_ptr(),
                                      _stream_handle(stream, pr.device)))
        return hv, (q.item() if q is not None else None)

    def backward(self, x=None, Ie=None, imea=None, grad_x=True, grad_Ie=True, stream=None):
        """(df/dx as (n, n) float32, df/dIe as (J,) float64); either may be None
        when not requested.  Recomputes the forward when it saved no state."""
        import torch
        pr = self.projector
        dev = "cuda:%d" % pr.device
        gx = torch.empty(pr.img_shape, dtype=torch.float32, device=dev) if grad_x else None
        gI = torch.empty(self.J, dtype=torch.float64, device=dev) if grad_Ie else None
        px, pI, pm = self._args(x, Ie, imea)
        check(lib().ctprj_bhc_backward(self._m, px, pI, pm,
                                       _dev_ptr(gx, pr.img_shape, pr.device) if gx is not None else None,
                                       _dptr(gI, self.J, torch.float64) if gI is not None else None,
                                       _stream_handle(stream, pr.device)))
        return gx, gI

    def spectrum_step(self, imea, Ie, newton_steps=2, stream=None):
        """FP64 Newton update of Ie >= 0 (in place, at most newton_steps steps)
        on the projections of the last saved forward; returns the likelihood
        at the returned Ie."""
        import torch
        f = ctypes.c_double()
        check(lib().ctprj_bhc_spectrum_step(self._m, _dptr(imea, self.nrays, torch.float32),
                                            _dptr(Ie, self.J, torch.float64), int(newton_steps),
                                            ctypes.byref(f), _stream_handle(stream, self.projector.device)))
        return f.value

    def reconstruct(self, x, Ie, imea, iterations, x_step=1.0, spectrum_newton_steps=2,
                    skip_spectrum=False, unfused=False, init_step="fixed", method="npg",
                    thresh=0.0, min_iterations=0, proximal="nonneg", u=0.0, max_inner=100,
                    admm_tol=1e-2, restart=True, adaptive_step=True, cumu_tol=4, wvlt_filter=None,
                    wvlt_levels=6, mask=None, wvlt_mask=None, pre_steps=2, stream=None):
        """The alternating density / spectrum loop, x and Ie updated in place.
        init_step: 'fixed' (first step x_step), 'bb' or 'hessian' (the
        reference's stepSizeInit rules); method: 'npg' (npg/NPG.m) or 'pg'
        (npg/PG.m) for the density step; thresh > 0 stops early by the
        reference's rule (relative density change <= thresh in three
        iterations after the first, more than min_iterations run);
        proximal: 'nonneg', 'tviso' or 'tvl1' (the reference's opt.proximal
        for NPG / PG), the TV maps with penalty weight u, a first inner
        iteration limit max_inner and a first inner tolerance scale admm_tol;
        restart, adaptive_step and cumu_tol are the reference's opt.restart,
        opt.adaptiveStep and opt.cumuTol.  proximal 'wvltADMM' (the reference's
        default) regularises with u |Psit(x)|_1 for the wavelet of scaling
        filter wvlt_filter (default daubcqf(2), Haar) and wvlt_levels levels.
        mask (n x n CUDA tensor, nonzero = reconstructed pixel) is the
        reference's opt.mask: the density lives on those pixels only;
        wvlt_mask is maskk, the coefficients of the masked transform (default:
        those the mask reaches, utils/wvltMask.m).  pre_steps is opt.preSteps
        (2, the BHC driver's default).
        Returns a dict with the cost after each iteration, the accepted density
        steps and the device time."""
        import torch
        pr = self.projector
        opts = LoopOpts(int(iterations), float(x_step), int(spectrum_newton_steps),
                        1 if skip_spectrum else 0, 1 if unfused else 0,
                        {"fixed": 0, "bb": 1, "hessian": 2}[init_step], {"npg": 0, "pg": 1}[method],
                        float(thresh), int(min_iterations),
                        {"nonneg": 0, "tviso": 1, "tvl1": 2, "wvltadmm": 3}[proximal.lower()], float(u),
                        int(max_inner), float(admm_tol), 0 if restart else 1, 0 if adaptive_step else 1,
                        int(cumu_tol))
        if wvlt_filter is not None:
            wf = np.asarray(wvlt_filter, np.float64)
            if wf.size > 20:
                raise ValueError("wavelet filters of at most 20 taps")
            opts.wvlt_filter_len = wf.size
            for j, v in enumerate(wf):
                opts.wvlt_filter[j] = float(v)
        opts.wvlt_levels = int(wvlt_levels)
        opts.pre_steps = int(pre_steps)
        keep = []
        for name, m in (("mask", mask), ("wvlt_mask", wvlt_mask)):
            if m is not None:
                mb = (m != 0).to(torch.uint8).contiguous()
                if mb.numel() != pr.img_shape[0] * pr.img_shape[1] or not mb.is_cuda:
                    raise ValueError("%s: expected an n x n CUDA tensor" % name)
                keep.append(mb)
                setattr(opts, name, mb.data_ptr())
        st = LoopStats()
        check(lib().ctprj_bhc_reconstruct(self._m, _dev_ptr(x, pr.img_shape, pr.device),
                                          _dptr(Ie, self.J, torch.float64),
                                          _dptr(imea, self.nrays, torch.float32), ctypes.byref(opts),
                                          ctypes.byref(st), _stream_handle(stream, pr.device)))
        n = min(st.iterations, len(st.cost))
        return {"iterations": st.iterations, "final_cost": st.final_cost, "ms": st.ms,
                "cost": list(st.cost[:n]), "x_step": list(st.x_step[:n]),
                "final_x_step": st.final_x_step, "ms_spectrum": st.ms_spectrum,
                "evaluations": st.evaluations, "restarts": st.restarts,
                "newton_steps": st.newton_steps, "converged": bool(st.converged),
                "x_change": list(st.x_change[:n]), "inner_iterations": st.inner_iterations,
                "prox_retries": st.prox_retries, "penalty": st.penalty}
