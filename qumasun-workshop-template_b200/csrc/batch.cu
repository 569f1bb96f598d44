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
// Each thread owns one grid column of its tile and marches z with the 9-deep
// column in registers; x and y neighbours come through the read-only data path
// (L1), so a tile reads its psi once from HBM plus its 4-wide halo.  Sums in the
// order of the per-system stencils (d = c0 p; d += x terms; d += y terms;
// d += z terms; out = V p + d), so FP32 keeps their rounding behaviour.
#include "qsb_internal.h"

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace {

constexpr int BTX = 32, BTY = 8, BNT = BTX * BTY;   // item tile and threads per CTA
constexpr int BZ = 32;                              // planes per item (z chunk)

template <typename T>
struct BSys {
    const T* in;
    T* out;
    const T* V;
    int nx, ny, nz;
    qsb::KC<T> k;
};

struct BItem {
    int sys, x0, y0, z0, band;
};

__device__ __forceinline__ int bwrap(int v, int n) {
    const int m = v % n;
    return m < 0 ? m + n : m;
}

template <typename T>
__global__ void __launch_bounds__(BNT) fd8_batch_kernel(const BSys<T>* __restrict__ sys, const BItem* __restrict__ items,
                                                         int n_items) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BItem w = items[it];
        const BSys<T> S = sys[w.sys];
        const int x = w.x0 + tx, y = w.y0 + ty;
        if (x >= S.nx || y >= S.ny) continue;
        const size_t nxy = (size_t)S.nx * S.ny;
        const size_t N = nxy * S.nz;
        const T* src = S.in + (size_t)w.band * N;
        T* dst = S.out + (size_t)w.band * N;
        const int z1 = min(S.nz, w.z0 + BZ);
        int xo[8], yo[8];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            xo[m] = bwrap(x - 4 + m, S.nx);
            xo[7 - m] = bwrap(x + 4 - m, S.nx);
            yo[m] = bwrap(y - 4 + m, S.ny) * S.nx;
            yo[7 - m] = bwrap(y + 4 - m, S.ny) * S.nx;
        }
        const size_t col = (size_t)y * S.nx + x;
        T q[9];   // z - 4 .. z + 4 of this column
#pragma unroll
        for (int m = 0; m < 8; ++m) q[m] = __ldg(src + (size_t)bwrap(w.z0 - 4 + m, S.nz) * nxy + col);
        for (int z = w.z0; z < z1; ++z) {
            q[8] = __ldg(src + (size_t)bwrap(z + 4, S.nz) * nxy + col);
            const T* pl = src + (size_t)z * nxy;
            const size_t row = (size_t)y * S.nx;
            const T xm4 = __ldg(pl + row + xo[0]), xm3 = __ldg(pl + row + xo[1]);
            const T xm2 = __ldg(pl + row + xo[2]), xm1 = __ldg(pl + row + xo[3]);
            const T xp4 = __ldg(pl + row + xo[7]), xp3 = __ldg(pl + row + xo[6]);
            const T xp2 = __ldg(pl + row + xo[5]), xp1 = __ldg(pl + row + xo[4]);
            const T ym4 = __ldg(pl + yo[0] + x), ym3 = __ldg(pl + yo[1] + x);
            const T ym2 = __ldg(pl + yo[2] + x), ym1 = __ldg(pl + yo[3] + x);
            const T yp4 = __ldg(pl + yo[7] + x), yp3 = __ldg(pl + yo[6] + x);
            const T yp2 = __ldg(pl + yo[5] + x), yp1 = __ldg(pl + yo[4] + x);
            const T p = q[4];
            const qsb::KC<T>& k = S.k;
            T d = k.c0 * p;
            d += k.cx[3] * (xp4 + xm4) + k.cx[2] * (xp3 + xm3) + k.cx[1] * (xp2 + xm2) + k.cx[0] * (xp1 + xm1);
            d += k.cy[3] * (yp4 + ym4) + k.cy[2] * (yp3 + ym3) + k.cy[1] * (yp2 + ym2) + k.cy[0] * (yp1 + ym1);
            d += k.cz[3] * (q[8] + q[0]) + k.cz[2] * (q[7] + q[1]) + k.cz[1] * (q[6] + q[2]) + k.cz[0] * (q[5] + q[3]);
            if constexpr (sizeof(T) == 4) d = fmaf(k.c0lo, p, d);
            dst[(size_t)z * nxy + col] = __ldg(S.V + (size_t)z * nxy + col) * p + d;
#pragma unroll
            for (int m = 0; m < 8; ++m) q[m] = q[m + 1];
        }
    }
}

template <typename T>
qsb_status launch_batch(int n, qsb_ham* const* hams, const int* nb, const void* const* psi, void* const* hpsi,
                        cudaStream_t s, int* launches) {
    std::vector<BSys<T>> hs(n);
    std::vector<BItem> items;
    std::vector<std::pair<long long, int>> order;   // (work, system): largest first
    for (int i = 0; i < n; ++i) {
        const qsb_ham* h = hams[i];
        hs[i] = BSys<T>{(const T*)psi[i], (T*)hpsi[i],
                        sizeof(T) == 8 ? (const T*)(const void*)h->V64 : (const T*)(const void*)h->V32, h->nx, h->ny,
                        h->nz, qsb::to_kc<T>(qsb::make_fd8_coef(-0.5, h->dx, h->dy, h->dz, 0, 0, 0))};
        order.push_back({(long long)h->N * nb[i], i});
    }
    std::sort(order.begin(), order.end(), [](const std::pair<long long, int>& a, const std::pair<long long, int>& b) {
        return a.first != b.first ? a.first > b.first : a.second < b.second;
    });
    for (const auto& o : order) {
        const int i = o.second;
        const qsb_ham* h = hams[i];
        for (int b = 0; b < nb[i]; ++b)
            for (int z0 = 0; z0 < h->nz; z0 += BZ)
                for (int y0 = 0; y0 < h->ny; y0 += BTY)
                    for (int x0 = 0; x0 < h->nx; x0 += BTX) items.push_back(BItem{i, x0, y0, z0, b});
    }
    if (items.empty()) return QSB_OK;
    if (items.size() > (size_t)0x7fffffff) return qsb::fail(QSB_ERR_INVALID, "ham_apply_batch: too many work items");
    // descriptors and the work list in one device block, freed once the launch is done
    const size_t sys_bytes = hs.size() * sizeof(BSys<T>);
    const size_t off_items = (sys_bytes + 255) / 256 * 256;
    const size_t bytes = off_items + items.size() * sizeof(BItem);
    void* dmem = nullptr;
    QSB_CUDA_TRY(cudaMallocAsync(&dmem, bytes, s));
    QSB_CUDA_TRY(cudaMemcpyAsync(dmem, hs.data(), sys_bytes, cudaMemcpyHostToDevice, s));
    QSB_CUDA_TRY(cudaMemcpyAsync((char*)dmem + off_items, items.data(), items.size() * sizeof(BItem),
                                 cudaMemcpyHostToDevice, s));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)std::min<size_t>(items.size(), (size_t)sms * 8);
    fd8_batch_kernel<T><<<grid, dim3(BTX, BTY), 0, s>>>((const BSys<T>*)dmem, (const BItem*)((char*)dmem + off_items),
                                                        (int)items.size());
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(dmem, s);
    if (e != cudaSuccess) return qsb::cuda_fail(e, "fd8_batch_kernel");
    ++*launches;
    // the host copies above are pageable: wait until they have been read
    QSB_CUDA_TRY(cudaStreamSynchronize(s));
    return QSB_OK;
}

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
    if (dtype == QSB_F64) QSB_TRY(launch_batch<double>(n_sys, hams, nb, psi, hpsi, s, &launches));
    else QSB_TRY(launch_batch<float>(n_sys, hams, nb, psi, hpsi, s, &launches));
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
