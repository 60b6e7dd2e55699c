// Step-by-step split solve of one volume, for callers that exchange halo
// columns between steps (column sharding over several GPUs).  FP32 state laid
// out with the mapping's own stride, so that a column's lines are the same
// span range in the state planes as in the mapping.  Included by
// potts_b200.cu inside its internal namespace.
#pragma once

}  // namespace

struct potts_stepper {
    potts_context *ctx = nullptr;
    MappingCopy mc;
    Geometry g{};
    DevBuf lines, state;  // state: Xi (3(K-1) planes), V (K-1), Vbar (K-1)
    int K = 0;
    float tau1 = 0.0f, tau2 = 0.0f, lambda = 0.0f;
    float c[POTTS_MAX_PHASES] = {};
    const float *d_u = nullptr;
};

namespace {

void stepper_free(potts_stepper *s)
{
    if (!s) return;
    if (s->ctx) {
        cudaSetDevice(s->ctx->device);
        cudaStreamSynchronize(s->ctx->stream);
    }
    for (DevBuf *d : {&s->lines, &s->state})
        if (d->p) cudaFree(d->p);
    delete s;
}

inline float *stepper_xi(potts_stepper *s) { return static_cast<float *>(s->state.p); }
inline float *stepper_v(potts_stepper *s) { return stepper_xi(s) + 3 * (size_t)(s->K - 1) * s->g.plane_w; }
inline float *stepper_vb(potts_stepper *s) { return stepper_v(s) + (size_t)(s->K - 1) * s->g.plane_w; }

template <int K>
PhaseParams<K> stepper_params(const potts_stepper *s)
{
    PhaseParams<K> pp;
    for (int i = 0; i < K; ++i) pp.c[i] = s->c[i];
    pp.lam = s->lambda;
    pp.tau1 = s->tau1;
    return pp;
}

// which: 0 init, 1 dual step, 2 primal step of iteration it, 3 argmax/outputs
template <int K>
int stepper_run(potts_stepper *s, int which, int it, float *res, uint8_t *labels, float *V)
{
    potts_context *ctx = s->ctx;
    if (s->g.n_lines == 0) return POTTS_OK;
    const unsigned nb = plain_blocks(s->g, 0, s->g.ns);
    cudaStream_t st = ctx->stream;
    switch (which) {
    case 0:
        POTTS_CUDA(cudaMemsetAsync(s->state.p, 0, s->state.bytes, st));
        potts::init_kernel<K, float><<<nb, potts::kPlainThreads, 0, st>>>(s->g, s->d_u, stepper_v(s), stepper_vb(s),
                                                                          stepper_params<K>(s));
        break;
    case 1:
        potts::dual_kernel<K, float><<<nb, potts::kPlainThreads, 0, st>>>(s->g, stepper_xi(s), stepper_vb(s), s->tau2,
                                                                          ctx->thr);
        break;
    case 2:
        potts::primal_kernel<K, float><<<nb, potts::kPlainThreads, 0, st>>>(
            s->g, stepper_xi(s), stepper_v(s), stepper_vb(s), s->d_u, stepper_params<K>(s), nullptr, it);
        break;
    default:
        potts::update_kernel<K, float><<<nb, potts::kPlainThreads, 0, st>>>(
            s->g, stepper_v(s), stepper_xi(s), stepper_params<K>(s), 0, s->g.ns, res, labels, V, nullptr,
            (int64_t)s->mc.span);
        break;
    }
    ctx->total_launches += 1;
    POTTS_CUDA(cudaGetLastError());
    return POTTS_OK;
}

int stepper_dispatch(potts_stepper *s, int which, int it, float *res, uint8_t *labels, float *V)
{
    if (!s) return fail(POTTS_EINVAL, "stepper is NULL");
    POTTS_CUDA(cudaSetDevice(s->ctx->device));
    switch (s->K) {
    case 2: return stepper_run<2>(s, which, it, res, labels, V);
    case 3: return stepper_run<3>(s, which, it, res, labels, V);
    case 4: return stepper_run<4>(s, which, it, res, labels, V);
    case 5: return stepper_run<5>(s, which, it, res, labels, V);
    case 6: return stepper_run<6>(s, which, it, res, labels, V);
    }
    return fail(POTTS_EINVAL, "K must be in [2, 6]");
}
