// Float64 geometry on the device: the child phases of every level and the final-stage direction cosines.
//
// Phases (fastsar/ffbp2.py:313-342 for the first two levels, fastsar/ffbp_cuda.py:598-632 below them): the range
// difference ddr between a child's centre and its parent's reference point, seen from the antenna at each input
// pulse, turned into the rotation phase at band centre (wrapped to [-0.5, 0.5] cycles) and its slope per frequency
// sample. The first two levels take the plain difference of the two distances, as the reference does on its host;
// the deeper levels take the reference's cancellation-free form num / (sqrt(wn^2 + num) + wn). Both run here in
// float64 once per plan, so a form call only reads the float32 results.
//
// Final geometry (fastsar/ffbp_cuda.py:870-886 and 964-975, fastsar/ffbp_cpu.py:187-199): per tile and final
// subaperture the unit vector from the tile centre to the antenna, along e1 and e2; per tile the aperture-mean
// unit vector (normalised) and the mean range, which set the quadratic phase correction.
#include "common.cuh"
#include "kernels.h"

namespace ffbp {

namespace {

__global__ void phases_kernel(const double *__restrict__ ant, int P, const double *__restrict__ ref, int Np,
                              const double *__restrict__ cen, int C, const double *__restrict__ range, double k0c,
                              double k1, int cancel_free, float2 *__restrict__ phase)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long total = (long)Np * C * P;
    if (idx >= total) return;
    const int p = (int)(idx % P);
    const long nc = idx / P;
    const int c = (int)(nc % C);
    const int n = (int)(nc / C);
    const double ax = ant[3 * p], ay = ant[3 * p + 1], az = ant[3 * p + 2];
    const double rx = ref[3 * n], ry = ref[3 * n + 1], rz = ref[3 * n + 2];
    double ddr;
    if (!cancel_free) {
        const double *q = cen + 3 * nc;                   // [Np, C, 3] centres
        const double cx = q[0] - ax, cy = q[1] - ay, cz = q[2] - az;
        double base;
        if (range) {
            base = range[p];
        } else {
            const double bx = rx - ax, by = ry - ay, bz = rz - az;
            base = sqrt(bx * bx + by * by + bz * bz);
        }
        ddr = sqrt(cx * cx + cy * cy + cz * cz) - base;
    } else {
        const double *d = cen + 3 * c;                    // [C, 3] offsets of the children from the parent's reference
        const double r = sqrt(ax * ax + ay * ay + az * az);
        const double ux = ax / r, uy = ay / r, uz = az / r;
        const double uc = rx * ux + ry * uy + rz * uz;
        const double rr = rx * rx + ry * ry + rz * rz;
        const double wn = r * sqrt(1.0 + (rr - 2.0 * r * uc) / (r * r));
        const double dx = d[0], dy = d[1], dz = d[2];
        const double ud = dx * ux + dy * uy + dz * uz;
        const double wd = r * ud - (dx * rx + dy * ry + dz * rz);
        const double num = (dx * dx + dy * dy + dz * dz) - 2.0 * wd;
        ddr = num / (sqrt(wn * wn + num) + wn);
    }
    const double cc = ddr * k0c;
    phase[idx] = make_float2((float)(cc - rint(cc)), (float)(ddr * k1));
}

__global__ void final_geom_kernel(const double *__restrict__ ant, int Pf, const double *__restrict__ cen, int B,
                                  double e1x, double e1y, double e1z, double e2x, double e2y, double e2z,
                                  double *__restrict__ ux, double *__restrict__ uy, double *__restrict__ ucx,
                                  double *__restrict__ ucy, double *__restrict__ rc)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const double enx = e1y * e2z - e1z * e2y, eny = e1z * e2x - e1x * e2z, enz = e1x * e2y - e1y * e2x;
    const double cx = cen[3 * b], cy = cen[3 * b + 1], cz = cen[3 * b + 2];
    double sx = 0.0, sy = 0.0, sz = 0.0, sr = 0.0;
    for (int p = 0; p < Pf; ++p) {
        const double wx = ant[3 * p] - cx, wy = ant[3 * p + 1] - cy, wz = ant[3 * p + 2] - cz;
        const double wn = sqrt(wx * wx + wy * wy + wz * wz);
        const double vx = (wx * e1x + wy * e1y + wz * e1z) / wn;
        const double vy = (wx * e2x + wy * e2y + wz * e2z) / wn;
        const double vz = (wx * enx + wy * eny + wz * enz) / wn;
        ux[(size_t)b * Pf + p] = vx;
        uy[(size_t)b * Pf + p] = vy;
        sx += vx; sy += vy; sz += vz; sr += wn;
    }
    sx /= Pf; sy /= Pf; sz /= Pf;
    const double mn = sqrt(sx * sx + sy * sy + sz * sz);
    ucx[b] = sx / mn;
    ucy[b] = sy / mn;
    rc[b] = sr / Pf;
}

}  // namespace

cudaError_t launch_phases(const double *ant, int P, const double *ref, int Np, const double *cen, int C,
                          const double *range, double k0c, double k1, int cancel_free, float2 *phase, cudaStream_t s)
{
    const long total = (long)Np * C * P;
    if (total <= 0) return cudaSuccess;
    const int nt = 256;
    const long nb = (total + nt - 1) / nt;
    phases_kernel<<<(unsigned)nb, nt, 0, s>>>(ant, P, ref, Np, cen, C, range, k0c, k1, cancel_free, phase);
    return cudaGetLastError();
}

cudaError_t launch_final_geom(const double *ant_f, int Pf, const double *cen, int B, const double *e1,
                              const double *e2, double *ux, double *uy, double *ucx, double *ucy, double *rc,
                              cudaStream_t s)
{
    if (B <= 0) return cudaSuccess;
    const int nt = 128;
    final_geom_kernel<<<(B + nt - 1) / nt, nt, 0, s>>>(ant_f, Pf, cen, B, e1[0], e1[1], e1[2], e2[0], e2[1], e2[2],
                                                       ux, uy, ucx, ucy, rc);
    return cudaGetLastError();
}

}  // namespace ffbp
