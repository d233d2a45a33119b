// The built-in reconstruction loop behind one call (the reference's compiled
// omegaMain entry, libHeader.h:1466, reconstructionAF.h:1053-1500, for the
// algorithms of this path): OSEM, OSL-OSEM, the relaxed ROSEM / RAMLA / BSREM /
// ROSEM-MAP / PKMA / MRAMLA / MBSREM for PET data, and PDHG with the smoothed
// TV gradient, with every
// sub-iteration issued on the caller's stream by the
// same entry points a custom loop uses, and (use_graph) one iteration captured
// as a CUDA graph and replayed.
#include <cmath>
#include <random>
#include <vector>

#include "kernels.h"

namespace omb {
namespace {

struct DevBuf {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
    float *f() const { return static_cast<float *>(p); }
};

int alloc(DevBuf &b, size_t bytes, cudaStream_t s) {
    b.s = s;
    OMB_CUDA_TRY(cudaMallocAsync(&b.p, bytes > 0 ? bytes : 4, s));
    return OMB_OK;
}

// Runs `body` n times: eagerly, or captured once as a graph and replayed.
template <class F>
int repeat(int n, bool use_graph, cudaStream_t s, F &&body) {
    if (!use_graph || n < 2 || s == nullptr) {
        for (int i = 0; i < n; ++i) {
            const int st = body();
            if (st != OMB_OK) return st;
        }
        return OMB_OK;
    }
    int st = body();  // warm-up outside the capture (lazy scratch allocations happen here)
    if (st != OMB_OK) return st;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    OMB_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    st = body();
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (st != OMB_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "graph capture of a reconstruction iteration");
    cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    for (int i = 1; i < n && e == cudaSuccess; ++i) e = cudaGraphLaunch(exec, s);
    if (exec) cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "graph replay of a reconstruction iteration");
    return OMB_OK;
}

}  // namespace
}  // namespace omb

using namespace omb;

extern "C" int omb_reconstruct(omb_handle *h, omb_recon_params *p, const float *y, const float *x0, float *x_out,
                               void *stream) {
    if (!h || !p) return set_error(OMB_ERR_INVALID, "handle/params pointer is NULL");
    if (p->struct_size != sizeof(omb_recon_params))
        return set_error(OMB_ERR_INVALID, "omb_recon_params.struct_size does not match this library");
    if (!y || !x0 || !x_out) return set_error(OMB_ERR_INVALID, "y/x0/x_out pointer is NULL");
    if (p->n_iter < 0) return set_error(OMB_ERR_INVALID, "n_iter must be >= 0");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = omb_image_count(h);
    if (n < 0) return -1;
    const int32_t n_subsets = handle_subsets(h);
    OMB_CUDA_TRY(cudaMemcpyAsync(x_out, x0, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    const bool graph = p->use_graph != 0;
    int st = OMB_OK;
    const int alg = p->algorithm;
    if (alg == OMB_RECON_PDHG_TV && p->tv_prox) {
        if (!(p->beta > 0.f)) return set_error(OMB_ERR_INVALID, "proximal TV needs beta > 0");
        if (p->diff_type != 0 && p->diff_type != 1) return set_error(OMB_ERR_INVALID, "diff_type must be 0 or 1");
    }
    if (alg == OMB_RECON_PDHG_TV && p->tgv) {
        if (p->tgv != 1 && p->tgv != 2) return set_error(OMB_ERR_INVALID, "tgv must be 0, 1 (3-D) or 2 (2-D)");
        if (p->tv_prox) return set_error(OMB_ERR_INVALID, "proximal TV and TGV exclude each other");
        if (!(p->alpha0_tgv > 0.f) || !(p->alpha1_tgv > 0.f))
            return set_error(OMB_ERR_INVALID, "TGV needs alpha0_tgv > 0 and alpha1_tgv > 0");
        if (p->diff_type != 0)
            return set_error(OMB_ERR_UNSUPPORTED, "TGV is built with forward differences only (diff_type 0)");
        if (!(p->beta >= 0.f)) return set_error(OMB_ERR_INVALID, "TGV needs beta >= 0");
    }
    if (alg == OMB_RECON_PDHG_TV || p->prior == OMB_PRIOR_TV) {
        if (p->tv_variant < OMB_TV_PLAIN || p->tv_variant > OMB_TV_APLS)
            return set_error(OMB_ERR_INVALID, "unknown TV variant");
        if (p->tv_variant >= OMB_TV_ANAT1 && !p->tv_ref)
            return set_error(OMB_ERR_INVALID, "anatomical TV and APLS need tv_ref");
    }
    if (alg >= OMB_RECON_OSEM && alg <= OMB_RECON_MBSREM && alg != OMB_RECON_PDHG_TV) {
        const bool osl = alg == OMB_RECON_OSL_OSEM;
        const bool map = alg == OMB_RECON_BSREM || alg == OMB_RECON_ROSEM_MAP;  // MAP step once per iteration
        const bool pkma = alg == OMB_RECON_PKMA;
        const bool mb = alg == OMB_RECON_MRAMLA || alg == OMB_RECON_MBSREM;
        const bool ramla = alg == OMB_RECON_RAMLA || alg == OMB_RECON_BSREM;    // no sensitivity image
        const bool relaxed = alg >= OMB_RECON_ROSEM;
        // the prior's gradient at every sub-iteration's image, added to the gradient (priors.h:361-370)
        const bool sub_prior = alg == OMB_RECON_MBSREM || (pkma && p->prior != 0);
        const bool need_prior = osl || map || sub_prior;
        const bool no_sens = ramla || pkma || mb;
        if (need_prior && (p->prior < OMB_PRIOR_RDP || p->prior > OMB_PRIOR_FMH))
            return set_error(OMB_ERR_INVALID, "unknown prior");
        if (need_prior && (p->prior == OMB_PRIOR_QUAD || p->prior == OMB_PRIOR_HUBER) && !p->prior_window)
            return set_error(OMB_ERR_INVALID, "the quadratic / Huber prior needs its window");
        if (need_prior && p->prior == OMB_PRIOR_WMEAN && !p->wmean_weights)
            return set_error(OMB_ERR_INVALID, "the weighted mean prior needs its weights");
        if (need_prior && p->prior == OMB_PRIOR_LFILTER && !p->lfilter_weights)
            return set_error(OMB_ERR_INVALID, "the L-filter prior needs its weights");
        if (need_prior && p->prior == OMB_PRIOR_FMH && !p->fmh_weights)
            return set_error(OMB_ERR_INVALID, "the FMH prior needs its weights");
        if (need_prior && p->prior == OMB_PRIOR_HYPERBOLIC && !p->hyper_weights)
            return set_error(OMB_ERR_INVALID, "the hyperbolic prior needs its weights");
        if (need_prior && p->prior == OMB_PRIOR_GGMRF && !p->ggmrf_weights)
            return set_error(OMB_ERR_INVALID, "the GGMRF prior needs its weights");
        if (need_prior && p->prior == OMB_PRIOR_NLM && !p->nlm_gaussian)
            return set_error(OMB_ERR_INVALID, "the NLM prior needs its patch weights");
        const Grid g = handle_grid(h);
        const float epps = handle_epps(h);
        // per-subset sensitivity images, then sub-iterations in subset order
        std::vector<int64_t> off(n_subsets + 1, 0);
        int64_t m_max = 0;
        for (int s_ = 0; s_ < n_subsets; ++s_) {
            const int64_t ms = omb_measurement_count(h, s_);
            off[s_ + 1] = off[s_] + ms;
            m_max = ms > m_max ? ms : m_max;
        }
        DevBuf sens, wm, wi, du, lam;
        if (!no_sens && (st = alloc(sens, (size_t)n_subsets * n * sizeof(float), s)) != OMB_OK) return st;
        if (need_prior && (st = alloc(du, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
        if ((st = alloc(wm, (size_t)m_max * sizeof(float), s)) != OMB_OK) return st;
        if ((st = alloc(wi, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
        Relax rl;
        Momentum mo;
        if (relaxed && p->n_iter > 0) {
            // lam[iter] (and PKMA's alpha[iter * S + subset]) in device memory with the iteration
            // counter behind them, so that a replayed iteration reads the next values
            // (libHeader.h:1331-1343; defaults prepass.py:962-972, 998-1006)
            const size_t nl = (size_t)p->n_iter, na = pkma ? (size_t)p->n_iter * n_subsets : 0;
            std::vector<float> host(nl + na + 1, 0.f);
            for (int i = 0; i < p->n_iter; ++i)
                host[i] = p->relaxation ? p->relaxation[i] : (float)(1.0 / (i / 20.0 + 1.0));
            for (size_t k = 0; k < na; ++k)
                host[nl + k] = p->momentum ? p->momentum[k] : (float)(1.0 + (0.45 * (double)k) / ((double)k + 100.0));
            if ((st = alloc(lam, host.size() * sizeof(float) + 16, s)) != OMB_OK) return st;
            int *counter = reinterpret_cast<int *>(lam.f() + host.size());
            OMB_CUDA_TRY(cudaMemcpyAsync(lam.p, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice, s));
            OMB_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int), s));
            // the host vector leaves scope: wait for the copy
            OMB_CUDA_TRY(cudaStreamSynchronize(s));
            rl.lam = lam.f();
            rl.iter = counter;
            if (pkma) {
                mo.alpha = lam.f() + nl;
                mo.iter = counter;
                mo.n_subsets = n_subsets;
            }
        }
        const float upper = p->upper_bound > 0.f ? p->upper_bound : 10000.f;
        // PKMA / MBSREM image preconditioner: D once, before the iterations
        DevBuf pd;
        if (p->precond < 0 || p->precond > 3 || (p->precond && !(pkma || mb)))
            return set_error(OMB_ERR_INVALID, "image preconditioners 1 to 3 are for PKMA / MRAMLA / MBSREM");
        const bool ifilt = p->img_filter_h != nullptr;
        const bool ext = p->precond == 3 || p->precond_alpha || p->precond_grad || p->precond_curv || ifilt;
        if ((ext || p->precond_meas) && !(pkma || mb))
            return set_error(OMB_ERR_INVALID, "the image and measurement preconditioners are for PKMA / MRAMLA / MBSREM");
        if (p->pkma_relax && !pkma) return set_error(OMB_ERR_INVALID, "the relaxation parameters are PKMA's");
        if (p->precond == 3 && !p->precond_ref)
            return set_error(OMB_ERR_INVALID, "image preconditioner type 2 needs precond_ref");
        if (p->precond_grad && (p->diff_type < 0 || p->diff_type > 2))
            return set_error(OMB_ERR_INVALID, "diff_type must be 0, 1 or 2");
        if (p->precond) {
            if ((st = alloc(pd, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
            if ((st = omb_precond_image(h, pd.f(), wi.f(), stream)) != OMB_OK) return st;
        }
        // the other preconditioners (functions.hpp:2057-2106, reconstructionAF.h:600-650, 827-861) and the
        // PKMA relaxation's workspace
        DevBuf ones, gradF, dP, alpha_d, meas_m, pwork, ftmp;
        if (ifilt) {
            if (p->img_filter_nf < g.nx || p->img_filter_nf < g.ny || p->img_filter_nf > 2048)
                return set_error(OMB_ERR_INVALID, "img_filter_nf must cover nx and ny (at most 2048)");
            if ((st = alloc(ftmp, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
        }
        if (p->precond_curv || p->precond_meas) {
            if ((st = alloc(ones, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
            OMB_CUDA_TRY(cudaMemsetAsync(ones.p, 0, (size_t)n * sizeof(float), s));
            if ((st = zero_to_one(ones.f(), n, s)) != OMB_OK) return st;  // an image of ones
        }
        if (p->precond_meas) {
            // A_s 1 of every subset, in subset order like y
            if ((st = alloc(meas_m, (size_t)off[n_subsets] * sizeof(float), s)) != OMB_OK) return st;
            for (int s_ = 0; s_ < n_subsets && st == OMB_OK; ++s_)
                st = omb_forward(h, s_, ones.f(), meas_m.f() + off[s_], stream);
            if (st == OMB_OK) st = zero_to_one(meas_m.f(), off[n_subsets], s);
            if (st != OMB_OK) return st;
        }
        if (p->precond_curv) {
            if ((st = alloc(dP, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
            for (int s_ = 0; s_ < n_subsets && st == OMB_OK; ++s_) {
                const int64_t ms = off[s_ + 1] - off[s_];
                st = omb_forward(h, s_, ones.f(), wm.f(), stream);
                if (st == OMB_OK) st = curv_meas(wm.f(), y + off[s_], ms, s);
                if (st == OMB_OK) st = omb_backward(h, s_, wm.f(), wi.f(), nullptr, OMB_BP_FLOAT_ATOMIC, stream);
                if (st == OMB_OK) st = curv_acc(dP.f(), wi.f(), n, n_subsets, s_ == 0, s);
            }
            if (st == OMB_OK) st = curv_finish(dP.f(), n, s);
            if (st != OMB_OK) return st;
        }
        if (p->precond_grad && (st = alloc(gradF, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
        if (p->precond_alpha) {
            const size_t na = (size_t)p->n_iter * n_subsets;
            if ((st = alloc(alpha_d, na * sizeof(float), s)) != OMB_OK) return st;
            OMB_CUDA_TRY(cudaMemcpyAsync(alpha_d.p, p->precond_alpha, na * sizeof(float), cudaMemcpyHostToDevice, s));
        }
        if ((ext || p->pkma_relax) &&
            (st = alloc(pwork, precond_workspace_bytes() + 2 * dot_workspace_bytes(), s)) != OMB_OK)
            return st;
        PrecondExt pe;
        pe.mode = p->precond;
        pe.dd = p->precond ? pd.f() : nullptr;
        pe.ref = p->precond_ref;
        pe.gradF = p->precond_grad ? gradF.f() : nullptr;
        pe.grad_init = p->grad_iters[0];
        pe.grad_last = p->grad_iters[1];
        pe.deriv_type = p->diff_type;
        pe.grad_v1 = p->grad_v[0];
        pe.grad_v2 = p->grad_v[1];
        pe.alpha = p->precond_alpha ? alpha_d.f() : nullptr;
        pe.dP = p->precond_curv ? dP.f() : nullptr;
        pe.it = rl.iter;
        pe.n_sub = n_subsets;
        pe.filt_h = p->img_filter_h;
        pe.filt_nf = p->img_filter_nf;
        pe.filt_K = p->filter_iters;
        pe.filt_tmp = ifilt ? ftmp.f() : nullptr;
        for (int s_ = 0; s_ < n_subsets && !no_sens && st == OMB_OK; ++s_)
            st = omb_sensitivity(h, s_, sens.f() + s_ * n, stream);
        if (st != OMB_OK) return st;
        // dU = beta * the prior's gradient at x_out
        auto prior_grad = [&]() -> int {
            if (cudaMemsetAsync(du.p, 0, (size_t)n * sizeof(float), s) != cudaSuccess)
                return set_error(OMB_ERR_CUDA, "clearing the prior gradient failed");
            if (p->prior == OMB_PRIOR_RDP)
                return omb_rdp_gradient_ex(x_out, du.f(), g.nx, g.ny, g.nz, p->rdp_gamma, epps, p->beta, p->rdp_edge,
                                           stream);
            if (p->prior == OMB_PRIOR_WMEAN)
                return omb_wmean_gradient(x_out, du.f(), g.nx, g.ny, g.nz, p->prior_g[0], p->prior_g[1], p->prior_g[2],
                                          p->wmean_weights, p->wmean_wsum > 0.f ? p->wmean_wsum : 1.f, p->wmean_type, epps,
                                          p->beta, p->mrp_no_norm, stream);
            if (p->prior == OMB_PRIOR_HYPERBOLIC)
                return omb_hyperbolic_gradient(x_out, du.f(), g.nx, g.ny, g.nz, p->prior_g[0], p->prior_g[1],
                                               p->prior_g[2], p->hyper_weights, p->hyper_delta, p->beta, stream);
            if (p->prior == OMB_PRIOR_GGMRF)
                return omb_ggmrf_gradient(x_out, du.f(), g.nx, g.ny, g.nz, p->prior_g[0], p->prior_g[1], p->prior_g[2],
                                          p->ggmrf_weights, p->ggmrf[0], p->ggmrf[1], p->ggmrf[2], p->beta, stream);
            if (p->prior == OMB_PRIOR_TV)
                return omb_tv_gradient_ex(x_out, du.f(), g.nx, g.ny, g.nz, p->beta, p->tv_smoothing, p->tv_variant,
                                          p->tv_sigma, p->tv_c, p->tv_ref, stream);
            if (p->prior == OMB_PRIOR_AD)
                return omb_ad_gradient(x_out, du.f(), g.nx, g.ny, g.nz, p->ad_dt, p->ad_k, p->ad_niter, p->ad_flux,
                                       p->ad_diffusion, epps, p->beta, p->mrp_no_norm, stream);
            if (p->prior == OMB_PRIOR_LFILTER)
                return omb_lfilter_gradient(x_out, du.f(), g.nx, g.ny, g.nz, p->prior_g[0], p->prior_g[1],
                                            p->prior_g[2], p->lfilter_weights, epps, p->beta, p->mrp_no_norm, stream);
            if (p->prior == OMB_PRIOR_FMH)
                return omb_fmh_gradient(x_out, du.f(), g.nx, g.ny, g.nz, p->prior_g[0], p->prior_g[1], p->prior_g[2],
                                        p->fmh_weights, epps, p->beta, p->mrp_no_norm, stream);
            if (p->prior == OMB_PRIOR_MRP)
                return omb_mrp_gradient(x_out, du.f(), g.nx, g.ny, g.nz, p->prior_g[0], p->prior_g[1], p->prior_g[2],
                                        epps, p->beta, p->mrp_no_norm, stream);
            if (p->prior == OMB_PRIOR_NLM)
                return omb_nlm_gradient(x_out, p->nlm_ref, du.f(), g.nx, g.ny, g.nz, p->prior_g, p->nlm_patch,
                                        p->nlm_gaussian, p->nlm_h, epps, p->beta, p->nlm_type, p->rdp_gamma, p->ggmrf,
                                        p->nlm_adaptive, p->nlm_adaptive_s, stream);
            // quadratic: the window applied at every voxel (priors.h:27-42); Huber clamps it
            int e = omb_psf_convolve(x_out, du.f(), g.nx, g.ny, g.nz, p->prior_window, p->prior_g[0], p->prior_g[1],
                                     p->prior_g[2], stream);
            if (e == OMB_OK)
                e = scale_clamp(du.f(), n, p->beta, p->prior == OMB_PRIOR_HUBER ? p->huber_delta : INFINITY, s);
            return e;
        };
        st = repeat(p->n_iter, graph, s, [&]() {
            int e = OMB_OK;
            for (int s_ = 0; s_ < n_subsets && e == OMB_OK; ++s_) {
                float *ss = no_sens ? nullptr : sens.f() + s_ * n;
                if (osl) {
                    // dU of the current image, then the one-step-late update
                    e = prior_grad();
                    if (e == OMB_OK) e = omb_osl_subset(h, s_, x_out, y + off[s_], ss, du.f(), wm.f(), wi.f(), stream);
                } else if (relaxed) {
                    RelaxedArgs ra;
                    ra.kind = pkma ? kPkma : (mb ? kMbsrem : (ramla ? kRamla : kRosem));
                    ra.sens = ss;
                    ra.lam = rl;
                    ra.alpha = mo;
                    ra.alpha.subset = s_;
                    ra.upper = upper;
                    ra.positivity = p->positivity != 0;
                    // with the other preconditioners on, precond_apply takes types 0-2 as well
                    ra.precond = ext ? 0 : p->precond;
                    ra.precond_d = p->precond && !ext ? pd.f() : nullptr;
                    ra.ext_on = ext;
                    ra.ext = pe;
                    ra.ext.sub = s_;
                    ra.gradF = p->precond_grad ? gradF.f() : nullptr;
                    ra.work = static_cast<double *>(pwork.p);
                    ra.meas_m = p->precond_meas ? meas_m.f() + off[s_] : nullptr;
                    ra.auto_relax = (p->pkma_relax & 1) != 0;
                    ra.relax_scaling = (p->pkma_relax & 2) != 0;
                    if (sub_prior) {
                        e = prior_grad();
                        ra.du = du.f();
                    }
                    if (e == OMB_OK) e = relaxed_subset(h, s_, x_out, y + off[s_], ra, wm.f(), wi.f(), s);
                } else {
                    e = omb_osem_subset(h, s_, x_out, y + off[s_], ss, wm.f(), wi.f(), stream);
                }
            }
            // BSREM / ROSEM-MAP: the prior at the iterate, then the MAP step (iterStep.h:14-34)
            if (e == OMB_OK && map) e = prior_grad();
            if (e == OMB_OK && map) e = map_step(x_out, du.f(), n, rl, epps, s);
            if (e == OMB_OK && relaxed) e = relax_advance(const_cast<int *>(rl.iter), s);
            return e;
        });
    } else if (p->algorithm == OMB_RECON_PDHG_TV) {
        const int64_t m_all = omb_measurement_count(h, -1);  // one subset: all measurements
        if (m_all < 0) return -1;
        const Grid g = handle_grid(h);
        DevBuf xn, u, pd, wm, wi, work, q, tr, tv;
        if ((st = alloc(xn, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
        if ((st = alloc(u, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
        if ((st = alloc(pd, (size_t)m_all * sizeof(float), s)) != OMB_OK) return st;
        if ((st = alloc(wm, (size_t)m_all * sizeof(float), s)) != OMB_OK) return st;
        if ((st = alloc(wi, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
        if (p->tv_prox) {
            // the proximal TV's dual variable, three images starting at zero
            if ((st = alloc(q, 3 * (size_t)n * sizeof(float), s)) != OMB_OK) return st;
            OMB_CUDA_TRY(cudaMemsetAsync(q.p, 0, 3 * (size_t)n * sizeof(float), s));
        }
        const bool tgv = p->tgv != 0;
        if (tgv) {
            // the TGV variables (functions.hpp:2936-2952): q 3 images, r 6 (3-D) or 3 (2-D), v 3 or 2, all zero
            const size_t nr = p->tgv == 1 ? 6 : 3, nv = p->tgv == 1 ? 3 : 2;
            if ((st = alloc(q, 3 * (size_t)n * sizeof(float), s)) != OMB_OK) return st;
            if ((st = alloc(tr, nr * (size_t)n * sizeof(float), s)) != OMB_OK) return st;
            if ((st = alloc(tv, nv * (size_t)n * sizeof(float), s)) != OMB_OK) return st;
            OMB_CUDA_TRY(cudaMemsetAsync(q.p, 0, 3 * (size_t)n * sizeof(float), s));
            OMB_CUDA_TRY(cudaMemsetAsync(tr.p, 0, nr * (size_t)n * sizeof(float), s));
            OMB_CUDA_TRY(cudaMemsetAsync(tv.p, 0, nv * (size_t)n * sizeof(float), s));
        }
        // the filtering-based measurement preconditioner (functions.hpp:2109-2166, computeForwardProject.h:
        // 21-45, 253-298): the residual filtered along the detector rows with h; while k < K the dual step is
        // p = (I + sigma F)^-1 (p + sigma F r) (the inverse filter hinv), afterwards the plain one without
        // filtering; with K = 0 every residual is filtered and the dual step stays the plain one
        const bool filt = p->filter_h != nullptr;
        // the filtering-based image preconditioner (functions.hpp:2093-2099, subiterStep.h:28-45): A^T p plus the
        // TV term filtered before the primal step in iterations k < K (K = 0: k = 0 only)
        const bool ifilt = p->img_filter_h != nullptr;
        if (filt && ifilt) return set_error(OMB_ERR_UNSUPPORTED, "one filtering-based preconditioner at a time");
        const int K = p->filter_iters;
        DevBuf wf, ftmp;
        if (ifilt) {
            if (p->img_filter_nf < g.nx || p->img_filter_nf < g.ny || p->img_filter_nf > 2048)
                return set_error(OMB_ERR_INVALID, "img_filter_nf must cover nx and ny (at most 2048)");
            if ((st = alloc(ftmp, (size_t)n * sizeof(float), s)) != OMB_OK) return st;
        }
        if (filt) {
            if (p->filter_rows < 1 || m_all % p->filter_rows != 0)
                return set_error(OMB_ERR_INVALID, "filter_rows must divide the measurement count");
            if (K > 0 && !p->filter_hinv) return set_error(OMB_ERR_INVALID, "filtering iterations need filter_hinv");
            if ((st = alloc(wf, (size_t)m_all * sizeof(float), s)) != OMB_OK) return st;
        }
        const int64_t fcols = filt ? m_all / p->filter_rows : 0;
        // power method (functions.hpp:2417-2540): x <- A^T (F) A x from an |N(0,1)| start normalised to unit
        // length (2430-2437); L = x . A^T (F) A x / x . x at the last step.  With the image filter P:
        // x <- P A^T A x in the power iterations it <= K (applyImagePreconditioning's kk <= filterIter)
        auto power = [&](bool use_filter, double &L) -> int {
            if (!work.p && (st = alloc(work, omb_power_workspace_bytes(), s)) != OMB_OK) return st;
            std::vector<float> v((size_t)n);
            std::mt19937 rng(1u);
            std::normal_distribution<float> nd(0.f, 1.f);
            double norm = 0.0;
            for (auto &a : v) {
                a = std::fabs(nd(rng));
                norm += (double)a * a;
            }
            const float inv = (float)(1.0 / std::sqrt(norm));
            for (auto &a : v) a *= inv;
            OMB_CUDA_TRY(cudaMemcpyAsync(xn.p, v.data(), (size_t)n * sizeof(float), cudaMemcpyHostToDevice, s));
            if (!use_filter) {
                const int e = omb_power_method(h, p->power_iterations > 0 ? p->power_iterations : 20, xn.f(), wm.f(),
                                               wi.f(), work.p, &L, stream);
                return e;
            }
            double *wl = static_cast<double *>(work.p);
            double *wn = wl + dot_workspace_bytes() / sizeof(double);
            const int iters = p->power_iterations > 0 ? p->power_iterations : 20;
            int e = OMB_OK;
            for (int it = 0; it < iters && e == OMB_OK; ++it) {
                e = omb_forward(h, -1, xn.f(), wm.f(), stream);
                if (e == OMB_OK && filt)
                    e = circ_filter(wm.f(), wf.f(), p->filter_rows, fcols, p->filter_h, p->filter_nf, s);
                if (e == OMB_OK) e = omb_backward(h, -1, filt ? wf.f() : wm.f(), wi.f(), nullptr, OMB_BP_FLOAT_ATOMIC,
                                                  stream);
                if (e == OMB_OK && ifilt && it <= K)
                    e = image_filter(wi.f(), ftmp.f(), g.nx, g.ny, g.nz, p->img_filter_h, p->img_filter_nf,
                                     FilterGate{}, s);
                if (e == OMB_OK && it == iters - 1) e = dot2(wi.f(), xn.f(), n, wl, s);
                if (e == OMB_OK) e = dot2(wi.f(), wi.f(), n, wn, s);
                if (e == OMB_OK) e = normalize_into(xn.f(), wi.f(), n, wn + dot_workspace_bytes() / sizeof(double) - 2, s);
            }
            if (e != OMB_OK) return e;
            double d[2];
            OMB_CUDA_TRY(cudaMemcpyAsync(d, wl + dot_workspace_bytes() / sizeof(double) - 2, sizeof(d),
                                         cudaMemcpyDeviceToHost, s));
            OMB_CUDA_TRY(cudaStreamSynchronize(s));
            L = d[0] / d[1];
            return OMB_OK;
        };
        float tau = p->tau;      // the step without filtering
        float tau_f = 0.f;       // the step while filtering
        if (filt) {
            tau_f = p->tau_filt;
            if (!(tau_f > 0.f)) {
                double L = 0.0;
                if ((st = power(true, L)) != OMB_OK) return st;
                if (!(L > 0.0)) return set_error(OMB_ERR_INVALID, "power method gave a non-positive eigenvalue");
                tau_f = (float)(1.0 / L);
            }
            if (!(tau > 0.f) && K > 0 && K < p->n_iter) {
                double L = 0.0;
                if ((st = power(false, L)) != OMB_OK) return st;
                if (!(L > 0.0)) return set_error(OMB_ERR_INVALID, "power method gave a non-positive eigenvalue");
                tau = (float)(1.0 / L);
            }
        } else if (ifilt) {
            // libHeader.h:1356-1361: tauCP is the step while filtering; the one after K comes from the power
            // method without the filter (functions.hpp:2696-2886)
            tau_f = p->tau;
            if (!(tau_f > 0.f)) {
                double L = 0.0;
                if ((st = power(true, L)) != OMB_OK) return st;
                if (!(L > 0.0)) return set_error(OMB_ERR_INVALID, "power method gave a non-positive eigenvalue");
                tau_f = (float)(1.0 / L);
            }
            if (K > 0 && K < p->n_iter) {
                double L = 0.0;
                if ((st = power(false, L)) != OMB_OK) return st;
                if (!(L > 0.0)) return set_error(OMB_ERR_INVALID, "power method gave a non-positive eigenvalue");
                tau = (float)(1.0 / L);
            }
        } else if (!(tau > 0.f)) {
            double L = 0.0;
            if ((st = power(false, L)) != OMB_OK) return st;
            if (!(L > 0.0)) return set_error(OMB_ERR_INVALID, "power method gave a non-positive eigenvalue");
            tau = (float)(1.0 / L);
        }
        p->tau_used = filt || ifilt ? tau_f : tau;
        p->tau_used2 = (filt || ifilt) && K > 0 && K < p->n_iter ? tau : 0.f;
        OMB_CUDA_TRY(cudaMemcpyAsync(u.p, x_out, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, s));
        OMB_CUDA_TRY(cudaMemsetAsync(pd.p, 0, (size_t)m_all * sizeof(float), s));
        // one iteration with steps tau_k, sig_k; fmode 0 no filtering, 1 filtered residual and the plain dual
        // step, 2 filtered residual and the inverse-filtered dual step.  The plain TV gradient is fused into
        // the primal step when nothing else comes between; the other TV terms are added to A^T p before it
        // the plain dual step divides by 1 + sigma, by 1 + sigma beta with TGV (computeForwardProject.h:295-303)
        auto one = [&](float *xa, float *xb, float tau_k, float sig_k, int fmode, bool imgf) {
            if (fmode == 0 && !imgf && !p->tv_prox && !tgv && p->tv_variant == OMB_TV_PLAIN)
                return omb_pdhg_iteration(h, xa, xb, u.f(), pd.f(), y, tau_k, sig_k, p->theta, p->beta,
                                          p->tv_smoothing, p->positivity, wm.f(), wi.f(), stream);
            const float denom = tgv ? 1.f + sig_k * p->beta : 1.f + sig_k;
            int e = omb_forward(h, -1, xa, wm.f(), stream);
            if (e == OMB_OK && fmode == 0 && !tgv) e = omb_pdhg_dual(pd.f(), wm.f(), y, m_all, sig_k, stream);
            if (e == OMB_OK && fmode == 0 && tgv) {
                e = meas_residual(wm.f(), y, m_all, s);
                if (e == OMB_OK) e = dual_step(pd.f(), wm.f(), pd.f(), m_all, sig_k, denom, s);
            }
            if (e == OMB_OK && fmode > 0) {
                e = meas_residual(wm.f(), y, m_all, s);
                if (e == OMB_OK) e = circ_filter(wm.f(), wf.f(), p->filter_rows, fcols, p->filter_h, p->filter_nf, s);
                if (e == OMB_OK && fmode == 1) e = dual_step(pd.f(), wf.f(), pd.f(), m_all, sig_k, denom, s);
                if (e == OMB_OK && fmode == 2) e = dual_step(pd.f(), wf.f(), wm.f(), m_all, sig_k, 1.f, s);
                if (e == OMB_OK && fmode == 2)
                    e = circ_filter(wm.f(), pd.f(), p->filter_rows, fcols, p->filter_hinv, p->filter_nf, s);
            }
            if (e == OMB_OK) e = omb_backward(h, -1, pd.f(), wi.f(), nullptr, OMB_BP_FLOAT_ATOMIC, stream);
            if (e == OMB_OK && tgv) {
                // priors.h:284-313: theta = thetaCP, tau the current primal step
                e = omb_proxtgv_step(xa, q.f(), tr.f(), tv.f(), wi.f(), g.nx, g.ny, g.nz, p->sigma2, p->alpha0_tgv,
                                     p->alpha1_tgv, p->theta, tau_k, p->l2_ball, p->tgv == 1, stream);
            } else if (e == OMB_OK && p->tv_prox) {
                // priors.h:261-281 between the backprojection and the primal step
                e = omb_proxtv_dual(xa, q.f(), g.nx, g.ny, g.nz, p->sigma2, p->beta, p->l2_ball, p->diff_type, stream);
                if (e == OMB_OK) e = omb_proxtv_divergence(q.f(), wi.f(), g.nx, g.ny, g.nz, p->diff_type, stream);
            } else if (e == OMB_OK) {
                e = omb_tv_gradient_ex(xa, wi.f(), g.nx, g.ny, g.nz, p->beta, p->tv_smoothing, p->tv_variant,
                                       p->tv_sigma, p->tv_c, p->tv_ref, stream);
            }
            if (e == OMB_OK && imgf)
                e = image_filter(wi.f(), ftmp.f(), g.nx, g.ny, g.nz, p->img_filter_h, p->img_filter_nf, FilterGate{},
                                 s);
            if (e == OMB_OK)
                e = omb_pdhg_primal(h, xa, wi.f(), u.f(), xb, tau_k, p->theta, 0.f, p->tv_smoothing, p->positivity,
                                    stream);
            return e;
        };
        if (!filt && !ifilt) {
            // two iterations per repetition keep x_out / xn in place for graph replays
            auto two = [&]() {
                int e = one(x_out, xn.f(), tau, p->sigma, 0, false);
                if (e == OMB_OK) e = one(xn.f(), x_out, tau, p->sigma, 0, false);
                return e;
            };
            st = repeat(p->n_iter / 2, graph, s, two);
            if (st == OMB_OK && p->n_iter % 2) {
                st = one(x_out, xn.f(), tau, p->sigma, 0, false);
                if (st == OMB_OK)
                    OMB_CUDA_TRY(cudaMemcpyAsync(x_out, xn.p, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, s));
            }
        } else {
            // the filter schedule changes at iteration K: eager iterations, host-side schedule
            float tau_k = tau_f, sig_k = p->sigma;
            float *xa = x_out, *xb = xn.f();
            for (int k = 0; k < p->n_iter && st == OMB_OK; ++k) {
                if (K > 0 && k == K) {
                    // computeForwardProject.h:22-35: the steps without filtering from here on
                    if (sig_k == 1.f) {
                        tau_k = tau;
                    } else if (sig_k == tau_k) {
                        tau_k = tau;
                        sig_k = tau;
                    } else {
                        sig_k = tau;
                    }
                }
                const int fmode = !filt ? 0 : (K > 0 ? (k < K ? 2 : 0) : 1);
                const bool imgf = ifilt && (K > 0 ? k < K : k == 0);
                st = one(xa, xb, tau_k, sig_k, fmode, imgf);
                std::swap(xa, xb);
            }
            if (st == OMB_OK && xa != x_out)
                OMB_CUDA_TRY(cudaMemcpyAsync(x_out, xa, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, s));
        }
    } else {
        return set_error(OMB_ERR_INVALID, "unknown reconstruction algorithm");
    }
    if (st != OMB_OK) return st;
    OMB_CUDA_TRY(cudaStreamSynchronize(s));
    return OMB_OK;
}
