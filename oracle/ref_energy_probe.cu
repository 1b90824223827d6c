// Probe around the reference's calcEnergy (pyGCMC gcmc/cpp/gcmc_energy.h:142-204)
// -- TEST INFRASTRUCTURE ONLY.
//
// Built by `make -C oracle ref` against the unmodified reference header (read
// where it lies), it evaluates the reference kernel's FP32 energy of explicit
// poses so the oracle can be pinned to the reference's own arithmetic.  One
// 128-thread block per pose, exactly as the reference's move kernels call it.
#include <cstdio>

#include "gcmc_energy.h"

extern "C" {

__global__ void ref_probe_kernel(const InfoStruct* info, AtomArray* frag, residue* res, Atom* atoms,
                                 const float* ff, const AtomArray* poses, const float* centres,
                                 float* out) {
    __shared__ InfoStruct SharedInfo;
    __shared__ AtomArray SharedFragmentInfo;
    __shared__ Atom tmp;
    if (threadIdx.x == 0) SharedInfo = info[0];
    if (threadIdx.x == 1) SharedFragmentInfo = poses[blockIdx.x];
    if (threadIdx.x == 2) {
        tmp.position[0] = centres[3 * blockIdx.x];
        tmp.position[1] = centres[3 * blockIdx.x + 1];
        tmp.position[2] = centres[3 * blockIdx.x + 2];
        tmp.charge = 0.0f;
        tmp.type = -1;
    }
    __syncthreads();
    calcEnergy(SharedInfo, SharedFragmentInfo, frag, res, atoms, ff, &tmp);
    __syncthreads();
    if (threadIdx.x == 0) out[blockIdx.x] = tmp.charge;
}

// poses[p]: an AtomArray whose atoms[] hold the pose's sites (positions,
// charges, types) and whose startRes is the residue to skip (-1 for none).
int ref_probe_energies(const InfoStruct* info, const AtomArray* frag, const residue* res,
                       const Atom* atoms, const float* ff, const AtomArray* poses,
                       const float* centres, int nposes, float* out) {
    InfoStruct* dI;
    AtomArray *dF, *dP;
    residue* dR;
    Atom* dA;
    float *dff, *dc, *dout;
    size_t nF = info->fragTypeNum, nR = info->totalResNum, nA = info->totalAtomNum;
    size_t nff = (size_t)info->ffXNum * info->ffYNum * 2;
    if (cudaMalloc(&dI, sizeof(InfoStruct)) || cudaMalloc(&dF, sizeof(AtomArray) * nF) ||
        cudaMalloc(&dR, sizeof(residue) * nR) || cudaMalloc(&dA, sizeof(Atom) * nA) ||
        cudaMalloc(&dff, sizeof(float) * nff) || cudaMalloc(&dP, sizeof(AtomArray) * nposes) ||
        cudaMalloc(&dc, sizeof(float) * 3 * nposes) || cudaMalloc(&dout, sizeof(float) * nposes))
        return 1;
    cudaMemcpy(dI, info, sizeof(InfoStruct), cudaMemcpyHostToDevice);
    cudaMemcpy(dF, frag, sizeof(AtomArray) * nF, cudaMemcpyHostToDevice);
    cudaMemcpy(dR, res, sizeof(residue) * nR, cudaMemcpyHostToDevice);
    cudaMemcpy(dA, atoms, sizeof(Atom) * nA, cudaMemcpyHostToDevice);
    cudaMemcpy(dff, ff, sizeof(float) * nff, cudaMemcpyHostToDevice);
    cudaMemcpy(dP, poses, sizeof(AtomArray) * nposes, cudaMemcpyHostToDevice);
    cudaMemcpy(dc, centres, sizeof(float) * 3 * nposes, cudaMemcpyHostToDevice);
    ref_probe_kernel<<<nposes, numThreadsPerBlock>>>(dI, dF, dR, dA, dff, dP, dc, dout);
    cudaError_t e = cudaDeviceSynchronize();
    cudaMemcpy(out, dout, sizeof(float) * nposes, cudaMemcpyDeviceToHost);
    cudaFree(dI); cudaFree(dF); cudaFree(dR); cudaFree(dA); cudaFree(dff); cudaFree(dP); cudaFree(dc);
    cudaFree(dout);
    return e == cudaSuccess ? 0 : 2;
}

}  // extern "C"
