// Differentiable solve: the forward pass keeps checkpoints of the state every
// `every` iterations; the backward pass recomputes each segment of iterations
// from its checkpoint (all states of the segment kept), then runs the
// reverse-mode kernels of kernels_adjoint.cuh through it, last iteration
// first.  Split schedule, FP32 state, one slab.  Included by potts_b200.cu
// inside its internal namespace.
#pragma once

}  // namespace

struct potts_tape {
    potts_context *ctx = nullptr;
    MappingCopy mc;
    Geometry g{};
    DevBuf lines, ckpt, seg, A, X, Q, P, grads, loss;
    int K = 0, iters = 0, every = 1, n_ckpt = 0;
    float tau1 = 0.0f, tau2 = 0.0f, lambda = 0.0f, eps = 0.0f;
    float c[POTTS_MAX_PHASES] = {};
    const float *d_u = nullptr;
    const uint8_t *d_truth = nullptr;
    double inv_count = 0.0;
};

namespace {

void tape_free(potts_tape *t)
{
    if (!t) return;
    if (t->ctx) {
        cudaSetDevice(t->ctx->device);
        cudaStreamSynchronize(t->ctx->stream);
    }
    for (DevBuf *d : {&t->lines, &t->ckpt, &t->seg, &t->A, &t->X, &t->Q, &t->P, &t->grads, &t->loss})
        if (d->p) cudaFree(d->p);
    delete t;
}

// One stored state: Xi (3(K-1) planes), V (K-1), Vbar (K-1).
struct TapeState {
    float *xi, *v, *vb;
};

inline size_t tape_state_floats(const potts_tape *t) { return 5 * (size_t)(t->K - 1) * (size_t)t->g.plane_w; }

inline TapeState tape_slot(const potts_tape *t, const DevBuf &buf, int i)
{
    float *base = static_cast<float *>(buf.p) + (size_t)i * tape_state_floats(t);
    const size_t pw = (size_t)t->g.plane_w;
    return TapeState{base, base + 3 * (size_t)(t->K - 1) * pw, base + 4 * (size_t)(t->K - 1) * pw};
}

template <int K>
PhaseParams<K> tape_params(const potts_tape *t)
{
    PhaseParams<K> pp;
    for (int i = 0; i < K; ++i) pp.c[i] = t->c[i];
    pp.lam = t->lambda;
    pp.tau1 = t->tau1;
    return pp;
}

template <int K>
int tape_iterate(potts_tape *t, const TapeState &s, int it)
{
    potts_context *ctx = t->ctx;
    const unsigned nb = plain_blocks(t->g, 0, t->g.ns);
    potts::dual_kernel<K, float><<<nb, potts::kPlainThreads, 0, ctx->stream>>>(t->g, s.xi, s.vb, t->tau2, ctx->thr);
    potts::primal_kernel<K, float><<<nb, potts::kPlainThreads, 0, ctx->stream>>>(t->g, s.xi, s.v, s.vb, t->d_u,
                                                                                 tape_params<K>(t), nullptr, it);
    ctx->total_launches += 2;
    POTTS_CUDA(cudaGetLastError());
    return POTTS_OK;
}

template <int K>
int tape_loss(potts_tape *t, const TapeState &final_state, double *loss)
{
    potts_context *ctx = t->ctx;
    const unsigned nb = plain_blocks(t->g, 0, t->g.ns);
    POTTS_CUDA(cudaMemsetAsync(t->loss.p, 0, sizeof(double), ctx->stream));
    potts::adj_loss_kernel<K><<<nb, potts::kPlainThreads, 0, ctx->stream>>>(
        t->g, final_state.v, t->d_truth, t->eps, t->inv_count, static_cast<float *>(t->A.p),
        static_cast<double *>(t->loss.p));
    ctx->total_launches += 1;
    POTTS_CUDA(cudaGetLastError());
    if (loss) {
        POTTS_CUDA(cudaMemcpyAsync(loss, t->loss.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        POTTS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return POTTS_OK;
}

template <int K>
int tape_forward(potts_tape *t, float *d_V, double *loss)
{
    potts_context *ctx = t->ctx;
    cudaStream_t s = ctx->stream;
    const size_t bytes = sizeof(float) * tape_state_floats(t);
    const TapeState run = tape_slot(t, t->seg, 0);
    const unsigned nb = plain_blocks(t->g, 0, t->g.ns);
    POTTS_CUDA(cudaMemsetAsync(t->seg.p, 0, bytes, s));
    potts::init_kernel<K, float><<<nb, potts::kPlainThreads, 0, s>>>(t->g, t->d_u, run.v, run.vb, tape_params<K>(t));
    ctx->total_launches += 1;
    POTTS_CUDA(cudaMemcpyAsync(tape_slot(t, t->ckpt, 0).xi, run.xi, bytes, cudaMemcpyDeviceToDevice, s));
    for (int it = 0; it < t->iters; ++it) {
        POTTS_TRY(tape_iterate<K>(t, run, it));
        const int k = it + 1;
        if (k % t->every == 0 || k == t->iters) {
            const int j = (k + t->every - 1) / t->every;
            POTTS_CUDA(cudaMemcpyAsync(tape_slot(t, t->ckpt, j).xi, run.xi, bytes, cudaMemcpyDeviceToDevice, s));
        }
    }
    if (d_V) {
        potts::update_kernel<K, float><<<nb, potts::kPlainThreads, 0, s>>>(
            t->g, run.v, run.xi, tape_params<K>(t), 0, t->g.ns, nullptr, nullptr, d_V, nullptr,
            (int64_t)t->mc.span);
        ctx->total_launches += 1;
    }
    return tape_loss<K>(t, run, loss);
}

template <int K>
int tape_backward(potts_tape *t, float *d_grad_u, double *grad_ci, double *grad_lambda)
{
    potts_context *ctx = t->ctx;
    cudaStream_t s = ctx->stream;
    const size_t bytes = sizeof(float) * tape_state_floats(t);
    const unsigned nb = plain_blocks(t->g, 0, t->g.ns);
    const int N = t->iters;
    POTTS_CUDA(cudaMemsetAsync(d_grad_u, 0, sizeof(float) * (size_t)t->mc.span, s));
    POTTS_CUDA(cudaMemsetAsync(t->X.p, 0, t->X.bytes, s));
    POTTS_CUDA(cudaMemsetAsync(t->P.p, 0, t->P.bytes, s));
    POTTS_CUDA(cudaMemsetAsync(t->grads.p, 0, t->grads.bytes, s));
    // dL/dV^N again, so that the backward pass can be repeated
    POTTS_TRY(tape_loss<K>(t, tape_slot(t, t->ckpt, t->n_ckpt - 1), nullptr));
    const PhaseParams<K> pp = tape_params<K>(t);
    for (int j = (N - 1) / t->every; j >= 0 && N > 0; --j) {
        const int k0 = j * t->every, k1 = std::min(k0 + t->every, N);
        POTTS_CUDA(cudaMemcpyAsync(tape_slot(t, t->seg, 0).xi, tape_slot(t, t->ckpt, j).xi, bytes,
                                   cudaMemcpyDeviceToDevice, s));
        for (int i = 0; i < k1 - k0; ++i) {
            const TapeState nxt = tape_slot(t, t->seg, i + 1);
            POTTS_CUDA(cudaMemcpyAsync(nxt.xi, tape_slot(t, t->seg, i).xi, bytes, cudaMemcpyDeviceToDevice, s));
            POTTS_TRY(tape_iterate<K>(t, nxt, k0 + i));
        }
        for (int k = k1 - 1; k >= k0; --k) {
            const TapeState sk = tape_slot(t, t->seg, k - k0), sk1 = tape_slot(t, t->seg, k - k0 + 1);
            potts::adj_primal_kernel<K><<<nb, potts::kPlainThreads, 0, s>>>(
                t->g, sk.v, sk1.xi, t->d_u, pp, t->tau2, static_cast<float *>(t->A.p),
                static_cast<const float *>(t->P.p), static_cast<float *>(t->Q.p), d_grad_u,
                static_cast<double *>(t->grads.p));
            potts::adj_dual_kernel<K><<<nb, potts::kPlainThreads, 0, s>>>(
                t->g, sk.xi, sk.vb, t->tau1, t->tau2, ctx->thr, static_cast<float *>(t->X.p),
                static_cast<const float *>(t->Q.p), static_cast<float *>(t->P.p));
            ctx->total_launches += 2;
        }
        POTTS_CUDA(cudaGetLastError());
    }
    double g[POTTS_MAX_PHASES + 1] = {};
    POTTS_CUDA(cudaMemcpyAsync(g, t->grads.p, sizeof(double) * (K + 1), cudaMemcpyDeviceToHost, s));
    POTTS_CUDA(cudaStreamSynchronize(s));
    if (grad_lambda) *grad_lambda = g[0];
    if (grad_ci)
        for (int i = 0; i < K; ++i) grad_ci[i] = g[1 + i];
    return POTTS_OK;
}

int tape_alloc(potts_tape *t)
{
    potts_context *ctx = t->ctx;
    const size_t state = sizeof(float) * tape_state_floats(t);
    const size_t pw = sizeof(float) * (size_t)t->g.plane_w;
    size_t free_b = 0, total_b = 0;
    POTTS_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t need = state * ((size_t)t->n_ckpt + (size_t)t->every + 1) +
                        pw * ((size_t)(t->K - 1) * 4 + (size_t)t->K * 4) + (size_t(256) << 20);
    if (need > free_b) return fail(POTTS_ENOMEM, "the checkpoints and the segment's states do not fit in memory");
    POTTS_TRY(ensure(ctx, t->ckpt, state * (size_t)t->n_ckpt));
    POTTS_TRY(ensure(ctx, t->seg, state * ((size_t)t->every + 1)));
    POTTS_TRY(ensure(ctx, t->A, pw * (size_t)(t->K - 1)));
    POTTS_TRY(ensure(ctx, t->X, pw * 3 * (size_t)(t->K - 1)));
    POTTS_TRY(ensure(ctx, t->Q, pw * (size_t)t->K));
    POTTS_TRY(ensure(ctx, t->P, pw * 3 * (size_t)t->K));
    POTTS_TRY(ensure(ctx, t->grads, sizeof(double) * (POTTS_MAX_PHASES + 1)));
    POTTS_TRY(ensure(ctx, t->loss, sizeof(double)));
    // the kernels read (and multiply by 0) neighbours outside the mask
    POTTS_CUDA(cudaMemsetAsync(t->Q.p, 0, t->Q.bytes, ctx->stream));
    return POTTS_OK;
}
