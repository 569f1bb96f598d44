// qsb_ham_apply_batch: H psi for many independent systems (different grids,
// band counts and projector sets) with the FD8 + V part of all of them in ONE
// persistent launch.
//
// The reference solves its systems one after another, each call a launch per
// operator piece; for a set of small, uneven cells (32^3 .. 64^3 grids, 8 .. 64
// bands) most of those launches leave most of the 148 SMs idle.  Here the
// stencil work of every system is cut into items (one 32 x 8 column tile of
// one band over a z chunk) in one list, balanced by size, and a persistent grid
// of a few CTAs per SM walks the list: the tail of one system overlaps the head
// of the next.  The nonlocal projection and expansion of each system keep their
// own launches (they are a fraction of the time at these sizes); the
// projections run before the batched stencil and the expansions after it, as
// in qsb_ham_apply.
//
// A persistent CTA runs, item after item, the tile work of the register-prefetch
// stencil (fd8_tile in stencil.cu: the tile plane with its 4-wide halo in a
// double-buffered shared tile, the z column of each thread's rows in
// registers, every global load issued planes ahead), so its arithmetic and
// summation order are those of the per-system FP32 stencil.
#include "qsb_internal.h"

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace {

// batched-or-not decisions of the autotuner, by the set's shape
std::mutex g_batch_mu;
std::map<std::vector<long long>, bool> g_batch_choice;

qsb_status apply_batched(qsb_dtype dtype, int n_sys, qsb_ham* const* hams, const int* nb, const void* const* psi,
                         void* const* hpsi, cudaStream_t s);

}  // namespace

extern "C" qsb_status qsb_ham_apply_batch(qsb_dtype dtype, int n_sys, qsb_ham* const* hams, const int* nb,
                                          const void* const* psi, void* const* hpsi, void* stream) {
    if (n_sys < 0 || (n_sys > 0 && (!hams || !nb || !psi || !hpsi)))
        return qsb::fail(QSB_ERR_INVALID, "ham_apply_batch: bad arguments");
    if (dtype != QSB_F64 && dtype != QSB_F32) return qsb::fail(QSB_ERR_INVALID, "ham_apply_batch: bad dtype");
    cudaStream_t s = (cudaStream_t)stream;
    for (int i = 0; i < n_sys; ++i) {
        QSB_TRY(qsb::check_apply(hams[i], dtype, nb[i], psi[i], hpsi[i]));
        if (!hams[i]->V64) return qsb::fail(QSB_ERR_STATE, "ham_apply_batch: potential not set on system " + std::to_string(i));
        if (hams[i]->kinetic != 0)
            return qsb::fail(QSB_ERR_INVALID, "ham_apply_batch: the batched stencil is the FD8 kinetic (system " +
                                                  std::to_string(i) + " is set to FFT)");
    }
    if (!qsb::autotune_enabled()) return apply_batched(dtype, n_sys, hams, nb, psi, hpsi, s);
    // autotuner: on the first call for this set of shapes, time the batched form
    // against the systems' own qsb_ham_apply, one after another, and keep the faster
    std::vector<long long> key{(long long)dtype, (long long)n_sys};
    for (int i = 0; i < n_sys; ++i) {
        key.push_back(hams[i]->nx);
        key.push_back(hams[i]->ny);
        key.push_back(hams[i]->nz);
        key.push_back(nb[i]);
    }
    bool batched = true, known = false;
    {
        std::lock_guard<std::mutex> g(g_batch_mu);
        auto it = g_batch_choice.find(key);
        if (it != g_batch_choice.end()) {
            known = true;
            batched = it->second;
        }
    }
    auto per_system = [&]() -> qsb_status {
        for (int i = 0; i < n_sys; ++i)
            QSB_TRY(qsb_ham_apply(hams[i], dtype, 0, nb[i], psi[i], hpsi[i], 0.0, 0.0, 0.0, stream));
        return QSB_OK;
    };
    if (!known) {
        cudaEvent_t e[3];
        for (auto& x : e) QSB_CUDA_TRY(cudaEventCreate(&x));
        QSB_TRY(apply_batched(dtype, n_sys, hams, nb, psi, hpsi, s));   // warm (and sizes workspaces)
        QSB_TRY(per_system());
        cudaEventRecord(e[0], s);
        QSB_TRY(apply_batched(dtype, n_sys, hams, nb, psi, hpsi, s));
        cudaEventRecord(e[1], s);
        QSB_TRY(per_system());
        cudaEventRecord(e[2], s);
        cudaEventSynchronize(e[2]);
        float tb = 0.f, tp = 0.f;
        cudaEventElapsedTime(&tb, e[0], e[1]);
        cudaEventElapsedTime(&tp, e[1], e[2]);
        for (auto& x : e) cudaEventDestroy(x);
        batched = tb <= tp;
        {
            std::lock_guard<std::mutex> g(g_batch_mu);
            g_batch_choice[key] = batched;
        }
        qsb::autotune_log("ham_apply_batch " + std::to_string(n_sys) + " systems: one persistent stencil launch " +
                          std::to_string(tb) + " ms, per-system applies " + std::to_string(tp) + " ms -> " +
                          (batched ? "batched" : "per system") + "\n");
    }
    return batched ? apply_batched(dtype, n_sys, hams, nb, psi, hpsi, s) : per_system();
}

namespace {

qsb_status apply_batched(qsb_dtype dtype, int n_sys, qsb_ham* const* hams, const int* nb, const void* const* psi,
                         void* const* hpsi, cudaStream_t s) {
    // 1) <beta|psi> of every system (each its own two launches)
    std::vector<double*> coef(n_sys, nullptr);
    int launches = 0;
    for (int i = 0; i < n_sys; ++i) {
        qsb_ham* h = hams[i];
        if (nb[i] == 0 || h->nl.n_points == 0) continue;
        const size_t need = qsb::nl_workspace_bytes(h->nl, nb[i]);
        if (need > h->ws_bytes) {
            if (h->ws) QSB_CUDA_TRY(cudaFree(h->ws));
            h->ws = nullptr;
            h->ws_bytes = 0;
            QSB_CUDA_TRY(cudaMalloc(&h->ws, need));
            h->ws_bytes = need;
        }
        QSB_TRY(qsb::nl_project(dtype, h->nl, h->nx, h->ny, h->nz, nb[i], 0, psi[i], h->dx * h->dy * h->dz, 0.0, 0.0,
                                0.0, false, h->ws, &coef[i], s));
        launches += 2;
    }
    // 2) V psi - 1/2 FD8 psi of all systems in one persistent launch
    std::vector<qsb::BatchSysDesc> d(n_sys);
    for (int i = 0; i < n_sys; ++i) {
        const qsb_ham* h = hams[i];
        d[i] = qsb::BatchSysDesc{psi[i], hpsi[i], dtype == QSB_F64 ? (const void*)h->V64 : (const void*)h->V32,
                                 h->nx, h->ny, h->nz, nb[i], qsb::make_fd8_coef(-0.5, h->dx, h->dy, h->dz, 0, 0, 0)};
    }
    QSB_TRY(qsb::launch_stencil_batch(dtype, n_sys, d.data(), s));
    ++launches;
    // 3) + the nonlocal expansion of every system
    for (int i = 0; i < n_sys; ++i) {
        if (!coef[i]) continue;
        qsb_ham* h = hams[i];
        QSB_TRY(qsb::nl_apply(dtype, h->nl, (int)h->N, nb[i], 0, hpsi[i], coef[i], 0.0, 0.0, 0.0, s));
        launches += 1;
    }
    return QSB_OK;
}

}  // namespace
