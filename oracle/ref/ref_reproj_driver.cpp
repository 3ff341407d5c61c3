// Test infrastructure only: a standalone driver around the reference's own
// projection-alignment re-projector (AreTomo3 AreTomo/ProjAlign/CCalcReproj
// + GReproj), compiled from the reference sources for sm_100a by
// oracle/ref/build_ref.sh into oracle/_ref/ref_reproj.  Parity target for the
// re-projection tests; nothing in the product links or calls it.
//
// Usage:
//   ref_reproj <in.bin> <out.bin> <volZ> <projIdx>
//
// in.bin : int32 nx, ny, T; float32 tilts_deg[T]; float32 frames[T][ny][nx]
// out.bin: int32 nx, ny; float32 reproj[ny][nx]
// As CProjAlignMain::mCalcReproj calls it (AreTomo/ProjAlign/
// CProjAlignMain.cpp:221-229): the projection being re-projected is marked
// skipped, every other one is not.
// stdout : one JSON line with the wall time of Setup + DoIt.
#include "AreTomo/ProjAlign/CProjAlignInc.h"
#include <cuda_runtime.h>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace MAP = McAreTomo::AreTomo::ProjAlign;

static bool read_all(FILE* f, void* p, size_t n) { return fread(p, 1, n, f) == n; }

int main(int argc, char** argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: %s in.bin out.bin volZ projIdx\n", argv[0]);
        return 2;
    }
    FILE* fi = fopen(argv[1], "rb");
    if (!fi) { perror("in"); return 3; }
    int hdr[3];
    if (!read_all(fi, hdr, sizeof(hdr))) return 3;
    const int nx = hdr[0], ny = hdr[1], nt = hdr[2];
    std::vector<float> tilts(nt);
    if (!read_all(fi, tilts.data(), sizeof(float) * nt)) return 3;
    std::vector<std::vector<float>> frames(nt, std::vector<float>((size_t)nx * ny));
    std::vector<float*> ptrs(nt);
    for (int t = 0; t < nt; t++) {
        if (!read_all(fi, frames[t].data(), sizeof(float) * (size_t)nx * ny)) return 3;
        ptrs[t] = frames[t].data();
    }
    fclose(fi);
    const int volZ = atoi(argv[3]), proj = atoi(argv[4]);
    std::vector<char> skip(nt, 0);
    skip[proj] = 1;
    float* out = nullptr;
    cudaMallocHost(&out, sizeof(float) * (size_t)nx * ny);
    cudaFree(0);  // create the context outside the timed region
    int stk[3] = {nx, ny, nt};
    auto t0 = std::chrono::steady_clock::now();
    {
        MAP::CCalcReproj calc;
        calc.Setup(stk, volZ, 0);
        calc.DoIt(ptrs.data(), tilts.data(), reinterpret_cast<bool*>(skip.data()), proj, out);
        cudaDeviceSynchronize();
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const cudaError_t err = cudaGetLastError();
    FILE* fo = fopen(argv[2], "wb");
    if (!fo) { perror("out"); return 4; }
    int ohdr[2] = {nx, ny};
    fwrite(ohdr, sizeof(int), 2, fo);
    fwrite(out, sizeof(float), (size_t)nx * ny, fo);
    fclose(fo);
    printf("{\"mode\": \"reproj\", \"nx\": %d, \"ny\": %d, \"tilts\": %d, \"volZ\": %d, \"proj\": %d, "
           "\"seconds\": %.6f, \"cuda\": \"%s\"}\n", nx, ny, nt, volZ, proj, secs, cudaGetErrorString(err));
    cudaFreeHost(out);
    return err == cudaSuccess ? 0 : 5;
}
