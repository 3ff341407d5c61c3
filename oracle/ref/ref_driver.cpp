// Test infrastructure only: a standalone driver around the reference's own
// CUDA Recon (AreTomo/Recon in AreTomo3), compiled from the reference sources
// in place by oracle/ref/build_ref.sh into oracle/_ref/ref_recon.  It is the
// parity target for the GPU tests; nothing in the product links or calls it.
//
// Usage:
//   ref_recon wbp  <in.bin> <out.bin> <volZ>
//   ref_recon sart <in.bin> <out.bin> <volZ> <startTilt> <numTilts> <iters> <subsets>
//
// in.bin : int32 nx, ny, T; float32 tilts_deg[T]; float32 frames[T][ny][nx]
// out.bin: int32 Nx, Nz, ny; float32 vol[ny][Nz][Nx]   (frames exactly as
//          CDoWbpRecon::DoIt / CDoSartRecon::DoIt return them: one XZ slice
//          per y, z already flipped by the reference)
// stdout : one JSON line with the wall time of the DoIt call.
// REF_FILL_SEED (environment, optional): the value time() returns, which
//          GGenRandoms::DoIt seeds the empty-voxel fill's random table with
//          (MaUtil/GGenRandoms.cu:42); unset, time() is the clock's.
#include "AreTomo/Recon/CReconInc.h"
#include "AreTomo/MrcUtil/CMrcUtilInc.h"
#include <cuda_runtime.h>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

namespace MAR = McAreTomo::AreTomo::Recon;

static long long g_seed = -1;
extern "C" time_t time(time_t* t)
{
    time_t v;
    if (g_seed >= 0) {
        v = (time_t)g_seed;
    } else {
        timespec ts{};
        clock_gettime(CLOCK_REALTIME, &ts);
        v = ts.tv_sec;
    }
    if (t) *t = v;
    return v;
}

static bool read_all(FILE* f, void* p, size_t n) { return fread(p, 1, n, f) == n; }

int main(int argc, char** argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: %s wbp|sart in.bin out.bin volZ [start num iters subsets]\n", argv[0]);
        return 2;
    }
    if (const char* e = getenv("REF_FILL_SEED")) g_seed = atoll(e);
    bool sart = strcmp(argv[1], "sart") == 0;
    if (sart && argc < 9) { fprintf(stderr, "sart needs 8 args\n"); return 2; }
    FILE* fi = fopen(argv[2], "rb");
    if (!fi) { perror("in"); return 3; }
    int hdr[3];
    if (!read_all(fi, hdr, sizeof(hdr))) { fprintf(stderr, "short header\n"); return 3; }
    int nx = hdr[0], ny = hdr[1], nt = hdr[2];
    std::vector<float> tilts(nt);
    if (!read_all(fi, tilts.data(), sizeof(float) * nt)) return 3;

    int stk[3] = {nx, ny, nt};
    MD::CTiltSeries* ts = new MD::CTiltSeries;
    ts->Create(stk);
    for (int t = 0; t < nt; t++) {
        if (!read_all(fi, ts->GetFrame(t), sizeof(float) * (size_t)nx * ny)) return 3;
        ts->m_pfTilts[t] = tilts[t];
    }
    fclose(fi);

    MAM::CAlignParam* aln = new MAM::CAlignParam;
    aln->Create(nt);
    for (int t = 0; t < nt; t++) aln->SetTilt(t, tilts[t]);

    int volZ = atoi(argv[4]);
    cudaFree(0);  // create the context outside the timed region
    auto t0 = std::chrono::steady_clock::now();
    MD::CTiltSeries* vol = nullptr;
    if (sart) {
        MAR::CDoSartRecon rec;
        vol = rec.DoIt(ts, aln, atoi(argv[5]), atoi(argv[6]), volZ, atoi(argv[7]), atoi(argv[8]));
    } else {
        MAR::CDoWbpRecon rec;
        vol = rec.DoIt(ts, aln, volZ);
    }
    cudaDeviceSynchronize();
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    cudaError_t err = cudaGetLastError();

    FILE* fo = fopen(argv[3], "wb");
    if (!fo) { perror("out"); return 4; }
    int ohdr[3] = {vol->m_aiStkSize[0], vol->m_aiStkSize[1], vol->m_aiStkSize[2]};
    fwrite(ohdr, sizeof(int), 3, fo);
    for (int y = 0; y < ohdr[2]; y++)
        fwrite(vol->GetFrame(y), sizeof(float), (size_t)ohdr[0] * ohdr[1], fo);
    fclose(fo);
    printf("{\"mode\": \"%s\", \"nx\": %d, \"ny\": %d, \"tilts\": %d, \"volZ\": %d, "
           "\"seconds\": %.6f, \"cuda\": \"%s\"}\n",
           sart ? "sart" : "wbp", nx, ny, nt, volZ, secs, cudaGetErrorString(err));
    delete vol;
    delete aln;
    delete ts;
    return err == cudaSuccess ? 0 : 5;
}
