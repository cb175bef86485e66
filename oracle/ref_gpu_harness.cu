/*
 * ref_gpu_harness.cu -- the reference's own MPD-RDME device functions,
 * compiled by nvcc for sm_100a, run on the B200.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile (target ref-gpu) into
 * oracle/_ref/ from the reference sources where they lie (nothing copied).
 * It serves two purposes:
 *   - the bit-exact authority for device arithmetic (CUDA's double exp in
 *     calculateReactionProbability, nvcc's default multiply-add contraction),
 *     compared against the C restatement and the product kernels;
 *   - the "reference kernels on B200" timing: refg_time runs the
 *     reference's per-timestep flow (x, y, z kernels, precomputed reaction
 *     kernel, cudaStreamSynchronize, mapped overflow-list check;
 *     MpdRdmeSolver.cu:996-1117).
 *
 * The kernel bodies are glue in the shape of mpd_{x,y,z}_kernel and
 * precomp_reaction_kernel (MpdRdmeSolver.cu:1342-1490, 1590-1675; the
 * 3-D-grid-launch build, options.cmake:55): they call the reference's
 * window loaders, choice, propagation and reaction functions in the same
 * order.  The precomputed propensity sum of :1613-1638 is restated.
 */
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "config.h"

#if defined(REF_BYTE)
#define MPD_WORDS_PER_SITE (MPD_LATTICE_MAX_OCCUPANCY / 4)
#elif defined(REF_INT)
#define MPD_WORDS_PER_SITE (MPD_LATTICE_MAX_OCCUPANCY)
#else
#error "define REF_BYTE or REF_INT"
#endif
#define MPD_APRON_SIZE 1

#include "cuda/constant.cu"
namespace refdev {
#include "rdme/dev/xor_random_dev.cu"
#include "rdme/dev/lattice_sim_1d_dev.cu"
#if defined(REF_BYTE)
#include "rdme/dev/byte_diffusion_1d_dev.cu"
#include "rdme/dev/byte_reaction_dev.cu"
#else
#include "rdme/dev/word_diffusion_1d_dev.cu"
#include "rdme/dev/word_reaction_dev.cu"
#endif
}  // namespace refdev
using namespace refdev;

static const unsigned REF_LIST_CAP_C = TUNE_MPD_MAX_PARTICLE_OVERFLOWS;
#include "ref_classic.h"

#if defined(REF_BYTE)
typedef uint8_t slot_t;
#else
typedef unsigned slot_t;
#endif

__global__ void __launch_bounds__(TUNE_MPD_X_BLOCK_MAX_X_SIZE, 1)
    gx_kernel(const unsigned *in, const uint8_t *st, unsigned *out, unsigned long long th, unsigned *list)
{
    const unsigned bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
    const unsigned lx = bx * blockDim.x + threadIdx.x;
    const unsigned li = bz * latticeXYSizeC + by * latticeXSizeC + lx;
    const unsigned wi = threadIdx.x + MPD_APRON_SIZE;
    __shared__ unsigned window[MPD_X_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    __shared__ uint8_t sitesWindow[MPD_X_WINDOW_SIZE];
    __shared__ unsigned choices[MPD_X_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    copyXWindowFromLattice(bx, in, window, li, lx, wi);
    copyXWindowFromSites(bx, st, sitesWindow, li, lx, wi);
    __syncthreads();
    makeXDiffusionChoices(window, sitesWindow, choices, li, lx, wi, blockDim.x, th);
    __syncthreads();
    performPropagation(out, window, choices, li, wi - 1, wi, wi + 1, MPD_X_WINDOW_SIZE, list);
}

__global__ void __launch_bounds__(TUNE_MPD_Y_BLOCK_X_SIZE *TUNE_MPD_Y_BLOCK_Y_SIZE, 1)
    gy_kernel(const unsigned *in, const uint8_t *st, unsigned *out, unsigned long long th, unsigned *list)
{
    const unsigned bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
    const unsigned ly = by * blockDim.y + threadIdx.y;
    const unsigned li = bz * latticeXYSizeC + ly * latticeXSizeC + bx * blockDim.x + threadIdx.x;
    const unsigned wy = threadIdx.y + MPD_APRON_SIZE, wi = wy * blockDim.x + threadIdx.x;
    __shared__ unsigned window[MPD_Y_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    __shared__ uint8_t sitesWindow[MPD_Y_WINDOW_SIZE];
    __shared__ unsigned choices[MPD_Y_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    copyYWindowFromLattice(in, window, li, ly, wi, wy);
    copyYWindowFromSites(st, sitesWindow, li, ly, wi, wy);
    __syncthreads();
    makeYDiffusionChoices(window, sitesWindow, choices, li, ly, wi, wy, th);
    __syncthreads();
    performPropagation(out, window, choices, li, wi - TUNE_MPD_Y_BLOCK_X_SIZE, wi, wi + TUNE_MPD_Y_BLOCK_X_SIZE,
                       MPD_Y_WINDOW_SIZE, list);
}

__global__ void __launch_bounds__(TUNE_MPD_Z_BLOCK_X_SIZE *TUNE_MPD_Z_BLOCK_Z_SIZE, 1)
    gz_kernel(const unsigned *in, const uint8_t *st, unsigned *out, unsigned long long th, unsigned *list)
{
    const unsigned bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
    const unsigned lz = bz * blockDim.z + threadIdx.z;
    const unsigned li = lz * latticeXYSizeC + by * latticeXSizeC + bx * blockDim.x + threadIdx.x;
    const unsigned wz = threadIdx.z + MPD_APRON_SIZE, wi = wz * blockDim.x + threadIdx.x;
    __shared__ unsigned window[MPD_Z_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    __shared__ uint8_t sitesWindow[MPD_Z_WINDOW_SIZE];
    __shared__ unsigned choices[MPD_Z_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    copyZWindowFromLattice(in, window, li, lz, wi, wz);
    copyZWindowFromSites(st, sitesWindow, li, lz, wi, wz);
    __syncthreads();
    makeZDiffusionChoices(window, sitesWindow, choices, li, lz, wi, wz, th);
    __syncthreads();
    performPropagation(out, window, choices, li, wi - TUNE_MPD_Z_BLOCK_X_SIZE, wi, wi + TUNE_MPD_Z_BLOCK_X_SIZE,
                       MPD_Z_WINDOW_SIZE, list);
}

__global__ void __launch_bounds__(TUNE_MPD_REACTION_BLOCK_X_SIZE *TUNE_MPD_REACTION_BLOCK_Y_SIZE, 1)
    gr_kernel(const unsigned *in, const uint8_t *st, unsigned *out, unsigned long long th, unsigned *list,
              const int8_t *SG, const uint8_t *RLG, const unsigned *ord, const unsigned *rsites, const unsigned *D1,
              const unsigned *D2, const float *rates, const float *qp0, const float *qp1, const float *qp2)
{
    const unsigned bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
    const unsigned ly = by * blockDim.y + threadIdx.y;
    const unsigned li = bz * latticeXYSizeC + ly * latticeXSizeC + bx * blockDim.x + threadIdx.x;
    unsigned particles[MPD_WORDS_PER_SITE];
    for (unsigned w = 0, off = 0; w < MPD_WORDS_PER_SITE; w++, off += latticeXYZSizeC) particles[w] = in[li + off];
    const uint8_t siteType = st[li];
    const slot_t *p = (const slot_t *)particles;
    float total = read_element(qp0, siteType);
    for (unsigned i = 0; i < MPD_LATTICE_MAX_OCCUPANCY; i++) {
        const slot_t p1 = p[i];
        if (p1 > 0) {
            total += read_element(qp1, siteType * numberSpeciesC + (p1 - 1));
            for (unsigned j = i + 1; j < MPD_LATTICE_MAX_OCCUPANCY; j++) {
                const slot_t p2 = p[j];
                if (p2 > 0)
                    total += read_element(qp2, siteType * numberSpeciesC * numberSpeciesC + (p1 - 1) * numberSpeciesC +
                                                   (p2 - 1));
            }
        }
    }
    if (total == 0.0f) return;
    const float prob = calculateReactionProbability(total);
    if (!checkForReaction(li, prob, th)) return;
#if defined(REF_BYTE)
    const unsigned idx =
        determineReactionIndex(siteType, (uint8_t *)particles, li, total, th, RLG, ord, rsites, D1, D2, rates);
    evaluateReaction(li, siteType, (uint8_t *)particles, idx, list, SG);
#else
    const unsigned idx = determineReactionIndex(siteType, particles, li, total, th, RLG, ord, rsites, D1, D2, rates);
    evaluateReaction(li, siteType, particles, idx, list, SG);
#endif
    for (unsigned w = 0, off = 0; w < MPD_WORDS_PER_SITE; w++, off += latticeXYZSizeC) out[li + off] = particles[w];
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

static unsigned g_X, g_Y, g_Z, g_ns, g_nst, g_nr;
static float *d_T, *d_qp0, *d_qp1, *d_qp2, *d_rate;
static unsigned *d_ord, *d_rsites, *d_D1, *d_D2;
static int8_t *d_S;
static uint8_t *d_RL;

#define RCK(x)                                                                       \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess) {                                                     \
            fprintf(stderr, "ref_gpu_harness: %s at %d\n", cudaGetErrorString(e_), __LINE__); \
            return -2;                                                               \
        }                                                                            \
    } while (0)

template <typename T>
static int upload(T **d, const T *h, size_t n)
{
    if (*d) cudaFree(*d);
    *d = nullptr;
    RCK(cudaMalloc(d, (n ? n : 1) * sizeof(T)));
    if (n) RCK(cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice));
    return 0;
}

extern "C" int refg_set_model(uint32_t X, uint32_t Y, uint32_t Z, uint32_t ns, uint32_t nst, uint32_t nr,
                              const float *T, const float *qp0, const float *qp1, const float *qp2,
                              const uint32_t *order, const uint32_t *D1, const uint32_t *D2, const float *rate,
                              const int8_t *S, const uint8_t *RL)
{
    g_X = X; g_Y = Y; g_Z = Z; g_ns = ns; g_nst = nst; g_nr = nr;
    std::vector<unsigned> rs(nr ? nr : 1, 0u);
    if (upload(&d_T, T, (size_t)nst * nst * ns) || upload(&d_qp0, qp0, nst) || upload(&d_qp1, qp1, (size_t)nst * ns) ||
        upload(&d_qp2, qp2, (size_t)nst * ns * ns) || upload(&d_rate, rate, nr) || upload(&d_ord, order, nr) ||
        upload(&d_rsites, rs.data(), nr) || upload(&d_D1, D1, nr) || upload(&d_D2, D2, nr) ||
        upload(&d_S, S, (size_t)nr * ns) || upload(&d_RL, RL, (size_t)nr * nst))
        return -2;
    // The symbols MpdRdmeSolver::buildModel / buildDiffusionModel set.
    const unsigned XY = X * Y, XYZ = X * Y * Z;
    RCK(cudaMemcpyToSymbol(numberReactionsC, &nr, sizeof(unsigned)));
    RCK(cudaMemcpyToSymbol(numberSpeciesC, &ns, sizeof(unsigned)));
    RCK(cudaMemcpyToSymbol(numberSiteTypesC, &nst, sizeof(unsigned)));
    RCK(cudaMemcpyToSymbol(latticeXSizeC, &X, sizeof(unsigned)));
    RCK(cudaMemcpyToSymbol(latticeYSizeC, &Y, sizeof(unsigned)));
    RCK(cudaMemcpyToSymbol(latticeZSizeC, &Z, sizeof(unsigned)));
    RCK(cudaMemcpyToSymbol(global_latticeZSizeC, &Z, sizeof(unsigned)));
    RCK(cudaMemcpyToSymbol(latticeXYSizeC, &XY, sizeof(unsigned)));
    RCK(cudaMemcpyToSymbol(latticeXYZSizeC, &XYZ, sizeof(unsigned)));
    RCK(cudaMemcpyToSymbol(global_latticeXYZSizeC, &XYZ, sizeof(unsigned)));
    RCK(cudaMemcpyToSymbol(TC, &d_T, sizeof(float *)));
    return 0;
}

/* MpdRdmeSolver.cu:1195-1261 launch geometry (3-D grid build). */
static void launch_step_kernel(int k, const unsigned *in, const uint8_t *st, unsigned *out, unsigned long long th,
                               unsigned *list, cudaStream_t s)
{
    if (k == 0) {
        unsigned bx = std::min((unsigned)TUNE_MPD_X_BLOCK_MAX_X_SIZE, g_X);
        if ((g_X / bx) * bx != g_X)
            for (unsigned t = 32; t < TUNE_MPD_X_BLOCK_MAX_X_SIZE; t += 32)
                if (g_X % t == 0) bx = t;
        gx_kernel<<<dim3(g_X / bx, g_Y, g_Z), dim3(bx, 1, 1), 0, s>>>(in, st, out, th, list);
    } else if (k == 1) {
        gy_kernel<<<dim3(g_X / TUNE_MPD_Y_BLOCK_X_SIZE, g_Y / TUNE_MPD_Y_BLOCK_Y_SIZE, g_Z),
                    dim3(TUNE_MPD_Y_BLOCK_X_SIZE, TUNE_MPD_Y_BLOCK_Y_SIZE, 1), 0, s>>>(in, st, out, th, list);
    } else if (k == 2) {
        gz_kernel<<<dim3(g_X / TUNE_MPD_Z_BLOCK_X_SIZE, g_Y, g_Z / TUNE_MPD_Z_BLOCK_Z_SIZE),
                    dim3(TUNE_MPD_Z_BLOCK_X_SIZE, 1, TUNE_MPD_Z_BLOCK_Z_SIZE), 0, s>>>(in, st, out, th, list);
    } else {
        gr_kernel<<<dim3(g_X / TUNE_MPD_REACTION_BLOCK_X_SIZE, g_Y / TUNE_MPD_REACTION_BLOCK_Y_SIZE, g_Z),
                    dim3(TUNE_MPD_REACTION_BLOCK_X_SIZE, TUNE_MPD_REACTION_BLOCK_Y_SIZE, 1), 0, s>>>(
            in, st, out, th, list, d_S, d_RL, d_ord, d_rsites, d_D1, d_D2, d_rate, d_qp0, d_qp1, d_qp2);
    }
}

/* The reference requires X % 32, Y % 8, Z % 8 (MpdRdmeSolver.cu:201-217). */
extern "C" int refg_supported(uint32_t X, uint32_t Y, uint32_t Z)
{
    return X % 32 == 0 && Y % TUNE_MPD_Y_BLOCK_Y_SIZE == 0 && Z % TUNE_MPD_Z_BLOCK_Z_SIZE == 0;
}

/*
 * Bit-exact replay: runs nsteps with a stream sync after every kernel so that
 * the overflow list can be split by phase and put in the canonical order
 * before the classic host reinsertion.  th[4*s+k]: timestep hashes.
 */
extern "C" int refg_run(uint32_t *lat, const uint8_t *sites, const uint64_t *th, uint32_t nsteps,
                        uint64_t *overflows_out)
{
    if (!refg_supported(g_X, g_Y, g_Z)) return -9;
    const size_t N = (size_t)g_X * g_Y * g_Z, bytes = N * REF_WORDS * 4;
    unsigned *d_a = nullptr, *d_b = nullptr, *list = nullptr;
    uint8_t *d_st = nullptr;
    RCK(cudaMalloc(&d_a, bytes));
    RCK(cudaMalloc(&d_b, bytes));
    RCK(cudaMalloc(&d_st, N));
    RCK(cudaHostAlloc(&list, (1 + 2 * REF_LIST_CAP_C) * sizeof(unsigned), cudaHostAllocMapped));
    unsigned *d_list = nullptr;
    RCK(cudaHostGetDevicePointer((void **)&d_list, list, 0));
    memset(list, 0, (1 + 2 * REF_LIST_CAP_C) * sizeof(unsigned));
    RCK(cudaMemcpy(d_a, lat, bytes, cudaMemcpyHostToDevice));
    RCK(cudaMemcpy(d_st, sites, N, cudaMemcpyHostToDevice));
    uint64_t ovf = 0;
    int rc = 0;
    for (uint32_t s = 0; s < nsteps && rc == 0; s++) {
        std::vector<Entry> entries;
        unsigned mark = 0;
        list[0] = 0;
        unsigned *src = d_a, *dst = d_b;
        for (int k = 0; k < 4; k++) {
            if (k == 3 && g_nr == 0) break;
            if (k < 3) {
                launch_step_kernel(k, src, d_st, dst, th[4 * s + k], d_list, 0);
                std::swap(src, dst);
            } else {
                launch_step_kernel(3, src, d_st, src, th[4 * s + 3], d_list, 0);
            }
            RCK(cudaDeviceSynchronize());
            const unsigned now = ((volatile unsigned *)list)[0];
            collect(list, mark, now, (unsigned)k, entries);
            mark = now;
        }
        // After three swaps the state is in `src`.
        if (src != d_a) std::swap(d_a, d_b);
        ovf += list[0];
        if (list[0] > REF_LIST_CAP_C) rc = -6;
        else if (list[0] > 0) {
            RCK(cudaMemcpy(lat, d_a, bytes, cudaMemcpyDeviceToHost));
            rc = classic_reinsert(lat, sites, entries, g_X, g_Y, g_Z);
            RCK(cudaMemcpy(d_a, lat, bytes, cudaMemcpyHostToDevice));
        }
    }
    RCK(cudaMemcpy(lat, d_a, bytes, cudaMemcpyDeviceToHost));
    cudaFree(d_a);
    cudaFree(d_b);
    cudaFree(d_st);
    cudaFreeHost(list);
    if (overflows_out) *overflows_out = ovf;
    return rc;
}

/*
 * The reference's timestep loop on the device: four launches, a stream sync
 * and a mapped overflow-list check per timestep (runTimestep,
 * MpdRdmeSolver.cu:996-1117).  Timesteps that overflow take the classic host
 * path.  *ms is the wall time of the loop.
 */
extern "C" int refg_time(uint32_t *lat, const uint8_t *sites, const uint64_t *th, uint32_t nsteps, double *ms)
{
    if (!refg_supported(g_X, g_Y, g_Z)) return -9;
    const size_t N = (size_t)g_X * g_Y * g_Z, bytes = N * REF_WORDS * 4;
    unsigned *d_a = nullptr, *d_b = nullptr, *list = nullptr, *d_list = nullptr;
    uint8_t *d_st = nullptr;
    cudaStream_t s;
    RCK(cudaStreamCreate(&s));
    RCK(cudaMalloc(&d_a, bytes));
    RCK(cudaMalloc(&d_b, bytes));
    RCK(cudaMalloc(&d_st, N));
    RCK(cudaHostAlloc(&list, (1 + 2 * REF_LIST_CAP_C) * sizeof(unsigned), cudaHostAllocMapped));
    RCK(cudaHostGetDevicePointer((void **)&d_list, list, 0));
    memset(list, 0, (1 + 2 * REF_LIST_CAP_C) * sizeof(unsigned));
    RCK(cudaMemcpy(d_a, lat, bytes, cudaMemcpyHostToDevice));
    RCK(cudaMemcpy(d_st, sites, N, cudaMemcpyHostToDevice));
    RCK(cudaDeviceSynchronize());
    int rc = 0;
    const auto t0 = std::chrono::steady_clock::now();
    for (uint32_t step = 0; step < nsteps && rc == 0; step++) {
        launch_step_kernel(0, d_a, d_st, d_b, th[4 * step + 0], d_list, s);
        launch_step_kernel(1, d_b, d_st, d_a, th[4 * step + 1], d_list, s);
        launch_step_kernel(2, d_a, d_st, d_b, th[4 * step + 2], d_list, s);
        std::swap(d_a, d_b);
        if (g_nr > 0) launch_step_kernel(3, d_a, d_st, d_a, th[4 * step + 3], d_list, s);
        RCK(cudaStreamSynchronize(s));
        const unsigned n = ((volatile unsigned *)list)[0];
        if (n > 0) {
            if (n > REF_LIST_CAP_C) {
                rc = -6;
                break;
            }
            std::vector<Entry> entries;
            collect(list, 0, n, 0, entries);
            RCK(cudaMemcpy(lat, d_a, bytes, cudaMemcpyDeviceToHost));
            rc = classic_reinsert(lat, sites, entries, g_X, g_Y, g_Z);
            RCK(cudaMemcpy(d_a, lat, bytes, cudaMemcpyHostToDevice));
            list[0] = 0;
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    RCK(cudaMemcpy(lat, d_a, bytes, cudaMemcpyDeviceToHost));
    cudaFree(d_a);
    cudaFree(d_b);
    cudaFree(d_st);
    cudaFreeHost(list);
    cudaStreamDestroy(s);
    return rc;
}
