// tex_probe.cu -- test helper: samples a float texture configured like the
// reference's micro-image textures (AdaptMIPMFrame.cpp:224-249: 32-bit float
// cudaArray, linear filtering, unnormalised coordinates, element-type reads)
// at (x + 0.5, y + 0.5), so that a test can compare the hardware's bilinear
// filtering with the engine's shared-memory emulation.  All fetch coordinates
// are finite; the texture unit bounds every fetch by its address mode.
#include <cuda_runtime.h>

__global__ void probe_kernel(cudaTextureObject_t tex, const float* xs, const float* ys, int n, float* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = tex2D<float>(tex, xs[i] + 0.5f, ys[i] + 0.5f);
}

extern "C" int tex_probe(const float* img, int w, int h, const float* xs, const float* ys, int n, int address_mode,
                         float* out)
{
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    float *d_x = nullptr, *d_y = nullptr, *d_o = nullptr;
    int rc = 0;
    cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    if (cudaMallocArray(&arr, &cd, w, h) != cudaSuccess) return -1;
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td = {};
    const cudaTextureAddressMode m = address_mode == 0 ? cudaAddressModeWrap : cudaAddressModeClamp;
    td.addressMode[0] = m;
    td.addressMode[1] = m;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    if (cudaMemcpy2DToArray(arr, 0, 0, img, w * sizeof(float), w * sizeof(float), h, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaCreateTextureObject(&tex, &rd, &td, nullptr) != cudaSuccess ||
        cudaMalloc(&d_x, n * sizeof(float)) != cudaSuccess || cudaMalloc(&d_y, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_o, n * sizeof(float)) != cudaSuccess ||
        cudaMemcpy(d_x, xs, n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_y, ys, n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = -2;
    } else {
        probe_kernel<<<(n + 255) / 256, 256>>>(tex, d_x, d_y, n, d_o);
        if (cudaMemcpy(out, d_o, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) rc = -3;
    }
    if (tex) cudaDestroyTextureObject(tex);
    cudaFreeArray(arr);
    cudaFree(d_x);
    cudaFree(d_y);
    cudaFree(d_o);
    return rc;
}
