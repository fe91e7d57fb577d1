// Stand-alone interstitial gather: the reference's hmlistln and olpistln
// (src/src_eigensystem/hmlistln.f90:61-86, olpistln.f90:53-82) as their own
// kernel.  The setup path fuses the same term (interstitial.cuh) into the
// contraction epilogue; this kernel serves callers that build the MT part
// elsewhere and is the HBM-bound form of the gather:
//   za(i, j) += V(ig) + 1/2 (k+G_i).(k+G_j) W(ig)        (H, i <= j)
//   za(i, j) += Theta(ig) [+ iora* term]                   (O, i <= j)
// with ig = ivgig(ivg(:, igpig(i)) - ivg(:, igpig(j))), only the upper
// triangle updated (Hermitianmatrix_indexedupdate, modfvsystem.f90:126-143).
// Bytes per upper element: read + write of H and O, 16 B each.
#include "exs_internal.cuh"
#include "interstitial.cuh"

namespace exs {

constexpr int IS_TILE = 32;

// One 32 x 32 tile of (i, j) per block (upper tiles only), 32 x 4 threads:
// thread x is the row i (coalesced along a column of za), y takes every
// fourth column j of the tile; the eight columns of a thread are loaded
// before any index lookup so that their DRAM reads overlap.  k-point
// blockIdx.z of the descriptor table (ngp, ld = nmat, igpig, vgpc, h, o).
constexpr int IS_TY = 4, IS_PER = IS_TILE / IS_TY;

__global__ void __launch_bounds__(128) interstitial_kernel(DevParams p, int which, const KDesc *ks)
{
    const KDesc kd = ks[blockIdx.z];
    const int bi = blockIdx.x, bj = blockIdx.y, ngp = kd.ngp;
    if (bi > bj || bj * IS_TILE >= ngp) return;
    __shared__ int siv[2][IS_TILE][3];
    __shared__ double sv[2][IS_TILE][3];
    const int tx = threadIdx.x, ty = threadIdx.y;
    if (ty < 2) {   // row (ty = 0) and column (ty = 1) G+k data of the tile (IS_TY >= 2)
        const int idx = (ty == 0 ? bi : bj) * IS_TILE + tx;
        if (idx < ngp) {
            int g = kd.igpig[idx] - 1;
            if (g < 0 || g >= p.ngrtot) {
                atomicOr(p.err, DEV_ERR_INDEX);
                g = 0;
            }
            for (int x = 0; x < 3; x++) {
                siv[ty][tx][x] = p.ivg[3 * g + x];
                sv[ty][tx][x] = kd.vgpc[3 * idx + x];
            }
        }
    }
    __syncthreads();
    const int i = bi * IS_TILE + tx;
    if (i >= ngp) return;
    const size_t ld = (size_t)kd.nmat;
    exs_complex hz[IS_PER], oz[IS_PER];
    bool ok[IS_PER];
#pragma unroll
    for (int q = 0; q < IS_PER; q++) {
        const int j = bj * IS_TILE + ty + IS_TY * q;
        ok[q] = j < ngp && i <= j;
        if (ok[q]) {
            const size_t e = (size_t)i + ld * j;
            if (which & 1) hz[q] = kd.h[e];
            if (which & 2) oz[q] = kd.o[e];
        }
    }
#pragma unroll
    for (int q = 0; q < IS_PER; q++) {
        if (!ok[q]) continue;
        const int jj = ty + IS_TY * q;
        const size_t e = (size_t)i + ld * (bj * IS_TILE + jj);
        double zr, zi;
        if ((which & 1) && interstitial(p, EPI_HAM, siv[0][tx], siv[1][jj], sv[0][tx], sv[1][jj], zr, zi)) {
            hz[q].re += zr;
            hz[q].im += zi;
            kd.h[e] = hz[q];
        }
        if ((which & 2) && interstitial(p, EPI_OVL, siv[0][tx], siv[1][jj], sv[0][tx], sv[1][jj], zr, zi)) {
            oz[q].re += zr;
            oz[q].im += zi;
            kd.o[e] = oz[q];
        }
    }
}

cudaError_t launch_interstitial(const DevParams &p, int which, const KDesc *d_k, int nk, int ngp_max, cudaStream_t s)
{
    if (nk <= 0 || ngp_max <= 0) return cudaSuccess;
    const int nt = (ngp_max + IS_TILE - 1) / IS_TILE;
    interstitial_kernel<<<dim3(nt, nt, nk), dim3(IS_TILE, IS_TY), 0, s>>>(p, which, d_k);
    return cudaGetLastError();
}

}  // namespace exs
