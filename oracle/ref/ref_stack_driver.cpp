// Test infrastructure only: a standalone driver around the reference's own
// input stage and thickness measurement, compiled from the reference sources
// for sm_100a by oracle/ref/build_ref.sh into oracle/_ref/ref_stack.  Parity
// target for the input-stage and thickness tests; nothing in the product
// links or calls it.
//
//   ref_stack stack <in.bin> <params.bin> <out.bin> <seed> <bin> <size_axis> [noaligned]
//     As CCorrTomoStack::DoIt / mCorrectProj run every tilt with Fourier
//     cropping (AreTomo/Correct/CCorrTomoStack.cpp:164-222): GCorrPatchShift
//     (shift, rotation, local patches, random fill) into the padded aligned
//     frame, then the forward 2-D FFT normalised, GFourierResize2D and the
//     inverse 2-D FFT of CFourierCropImage::mCropFFT (or its mCopy when the
//     sizes agree), unpadded.  The fill's random table is seeded with `seed`:
//     this driver defines time() to return it, which GGenRandoms::DoIt reads.
//     `noaligned` skips the copy-out of the aligned frames (not part of
//     CCorrTomoStack::DoIt), for timing; out.bin then has no aligned block.
//     in.bin    : int32 nx, ny, T; float32 tilts[T]; float32 frames[T][ny][nx]
//     params.bin: int32 P, shift_only; float32 shifts[T][2]; float32 axes[T];
//                 float32 local[T][5][P]
//     out.bin   : int32 ax, ay, bx, by; float32 aligned[T][ay][ax];
//                 float32 binned[T][by][bx]; int32 n; int32 table[n] (the
//                 fill's random table GGenRandoms drew)
//
//   ref_stack thick <vol.bin> <out.bin> <bin>
//     CCalcVolThick's measurement on a given flipped volume
//     (CCalcVolThick.cpp:85-106): mSetup, mMeasureStd of every plane,
//     mSmooth, mDetectEdges, called on the reference's own object.
//     vol.bin: int32 Nx, ny, Nz; float32 vol[Nz][ny][Nx] (FlipVol(true) frames)
//     out.bin: int32 n, e0, e1, thickness, offset_z; float32 raw[n]; float32 smoothed[n]
//
// stdout: one JSON line.
#include <cuda_runtime.h>
#include <cufft.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

// the reference's private members are reached from this driver only
#define private public
#include "AreTomo/Correct/CCorrectInc.h"
#include "AreTomo/MrcUtil/CMrcUtilInc.h"
#include "AreTomo/Recon/CReconInc.h"
#include "MaUtil/CMaUtilInc.h"
#undef private

namespace MAC = McAreTomo::AreTomo::Correct;
namespace MAR = McAreTomo::AreTomo::Recon;
namespace MAM = McAreTomo::AreTomo::MrcUtil;
namespace MU = McAreTomo::MaUtil;
namespace MD = McAreTomo::DataUtil;

static time_t g_seed = 0;
extern "C" time_t time(time_t* t)
{
    if (t) *t = g_seed;
    return g_seed;
}

static bool read_all(FILE* f, void* p, size_t n) { return fread(p, 1, n, f) == n; }

static int run_stack(int argc, char** argv)
{
    if (argc < 8) return 2;
    FILE* fi = fopen(argv[2], "rb");
    if (!fi) return 3;
    int hdr[3];
    if (!read_all(fi, hdr, sizeof(hdr))) return 3;
    const int nx = hdr[0], ny = hdr[1], nt = hdr[2];
    std::vector<float> tilts(nt);
    std::vector<float> raw((size_t)nt * nx * ny);
    if (!read_all(fi, tilts.data(), sizeof(float) * nt) || !read_all(fi, raw.data(), sizeof(float) * raw.size()))
        return 3;
    fclose(fi);
    FILE* fp = fopen(argv[3], "rb");
    if (!fp) return 3;
    int ph[2];
    if (!read_all(fp, ph, sizeof(ph))) return 3;
    const int P = ph[0], shift_only = ph[1];
    std::vector<float> shifts(2 * nt), axes(nt), local((size_t)nt * 5 * std::max(P, 0));
    if (!read_all(fp, shifts.data(), sizeof(float) * shifts.size()) ||
        !read_all(fp, axes.data(), sizeof(float) * axes.size()) ||
        (P > 0 && !read_all(fp, local.data(), sizeof(float) * local.size())))
        return 3;
    fclose(fp);
    g_seed = (time_t)strtoll(argv[5], nullptr, 10);
    const float bin = (float)atof(argv[6]), size_axis = (float)atof(argv[7]);
    const bool keep_aligned = !(argc > 8 && std::string(argv[8]) == "noaligned");

    int raw_size[2] = {nx, ny}, aln[2] = {0, 0}, bnd[2] = {0, 0};
    MAC::CCorrectUtil::CalcAlignedSize(raw_size, size_axis, aln);
    MAC::CCorrectUtil::CalcBinnedSize(aln, bin, true, bnd);
    int aln_pad[2] = {(aln[0] / 2 + 1) * 2, aln[1]};
    int bin_pad[2] = {(bnd[0] / 2 + 1) * 2, bnd[1]};
    float *g_raw = nullptr, *g_corr = nullptr, *g_bin = nullptr, *g_local = nullptr;
    cudaMalloc(&g_raw, sizeof(float) * nx * ny);
    cudaMalloc(&g_corr, sizeof(float) * aln_pad[0] * aln_pad[1]);
    cudaMalloc(&g_bin, sizeof(float) * (size_t)std::max(bin_pad[0] * bin_pad[1], aln_pad[0] * aln_pad[1]));
    cudaMemset(g_corr, 0, sizeof(float) * aln_pad[0] * aln_pad[1]);
    if (P > 0) cudaMalloc(&g_local, sizeof(float) * 5 * P);
    std::vector<float> aligned(keep_aligned ? (size_t)nt * aln[0] * aln[1] : 0), binned((size_t)nt * bnd[0] * bnd[1]);
    std::vector<int> table;
    cudaDeviceSynchronize();
    auto t0 = std::chrono::steady_clock::now();
    {
        MAC::GCorrPatchShift corr;
        corr.SetSizes(raw_size, false, aln_pad, true, P);
        {
            MU::GGenRandoms* gen = corr.m_pFillEmpty2D->m_pGenRandoms;
            table.resize(gen->m_iSize);
            cudaMemcpy(table.data(), gen->m_giRandoms, sizeof(int) * table.size(), cudaMemcpyDefault);
        }
        MU::CCufft2D fwd, inv;
        MU::CPad2D pad;
        const bool same = aln[0] == bnd[0] && aln[1] == bnd[1];
        for (int t = 0; t < nt; t++) {
            cudaMemcpy(g_raw, raw.data() + (size_t)t * nx * ny, sizeof(float) * nx * ny, cudaMemcpyDefault);
            if (P > 0) cudaMemcpy(g_local, local.data() + (size_t)t * 5 * P, sizeof(float) * 5 * P, cudaMemcpyDefault);
            // the column an odd aligned width leaves unwritten reads 0 here, as in the product
            cudaMemset(g_corr, 0, sizeof(float) * aln_pad[0] * aln_pad[1]);
            float shift[2] = {shifts[2 * t], shifts[2 * t + 1]};
            const float axis = shift_only ? 0.0f : axes[t];
            corr.DoIt(g_raw, shift, axis, g_local, true, g_corr);
            if (keep_aligned) pad.Unpad(g_corr, aln_pad, aligned.data() + (size_t)t * aln[0] * aln[1]);
            if (same) {
                pad.Unpad(g_corr, aln_pad, binned.data() + (size_t)t * bnd[0] * bnd[1]);
                continue;
            }
            // CFourierCropImage::mCropFFT
            fwd.CreateForwardPlan(aln, false);
            inv.CreateInversePlan(bnd, false);
            fwd.Forward(g_corr, true);
            int cmp_in[2] = {aln[0] / 2 + 1, aln[1]}, cmp_out[2] = {bnd[0] / 2 + 1, bnd[1]};
            MU::GFourierResize2D resize;
            resize.DoIt((cufftComplex*)g_corr, cmp_in, (cufftComplex*)g_bin, cmp_out, false);
            inv.Inverse((cufftComplex*)g_bin);
            pad.Unpad(g_bin, bin_pad, binned.data() + (size_t)t * bnd[0] * bnd[1]);
        }
        cudaDeviceSynchronize();
    }
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const cudaError_t err = cudaGetLastError();
    FILE* fo = fopen(argv[4], "wb");
    if (!fo) return 4;
    int oh[4] = {aln[0], aln[1], bnd[0], bnd[1]};
    fwrite(oh, sizeof(int), 4, fo);
    fwrite(aligned.data(), sizeof(float), aligned.size(), fo);
    fwrite(binned.data(), sizeof(float), binned.size(), fo);
    const int ntab = (int)table.size();
    fwrite(&ntab, sizeof(int), 1, fo);
    fwrite(table.data(), sizeof(int), table.size(), fo);
    fclose(fo);
    printf("{\"mode\": \"stack\", \"seconds\": %.6f, \"aligned\": [%d, %d], \"binned\": [%d, %d], \"cuda\": \"%s\"}\n",
           sec, aln[0], aln[1], bnd[0], bnd[1], cudaGetErrorString(err));
    cudaFree(g_raw);
    cudaFree(g_corr);
    cudaFree(g_bin);
    if (g_local) cudaFree(g_local);
    return err == cudaSuccess ? 0 : 5;
}

static int run_thick(int argc, char** argv)
{
    if (argc < 5) return 2;
    FILE* fi = fopen(argv[2], "rb");
    if (!fi) return 3;
    int hdr[3];
    if (!read_all(fi, hdr, sizeof(hdr))) return 3;
    const int Nx = hdr[0], ny = hdr[1], nz = hdr[2];
    MAM::CAlignParam::CreateInstances(1);
    MD::CTiltSeries* vol = new MD::CTiltSeries;
    int stk[3] = {Nx, ny, nz};
    vol->Create(stk);
    for (int z = 0; z < nz; z++)
        if (!read_all(fi, vol->GetFrame(z), sizeof(float) * (size_t)Nx * ny)) return 3;
    fclose(fi);
    MAR::CCalcVolThick calc;
    calc.m_pVolSeries = vol;
    calc.m_fBinning = (float)atof(argv[4]);
    calc.m_iNthGpu = 0;
    calc.m_aiSampleEdges[0] = calc.m_aiSampleEdges[1] = 0;
    calc.mSetup();
    // CCalcVolThick::DoIt, lines 97-106
    int start[2] = {0};
    start[0] = (calc.m_pVolSeries->m_aiStkSize[0] - calc.m_aiTileSize[0]) / 2;
    start[1] = (calc.m_pVolSeries->m_aiStkSize[1] - calc.m_aiTileSize[1]) / 2;
    const int n = calc.m_pVolSeries->m_aiStkSize[2] - 1;
    std::vector<float> cc(n), raw_cc(n);
    for (int z = 0; z < n; z++) cc[z] = calc.mMeasureStd(z, start);
    raw_cc = cc;
    calc.mSmooth(cc.data(), n);
    calc.mDetectEdges(cc.data(), n);
    MAM::CAlignParam* aln = MAM::CAlignParam::GetInstance(0);
    int oh[5] = {n, calc.m_aiSampleEdges[0], calc.m_aiSampleEdges[1], aln->m_iThickness, aln->m_iOffsetZ};
    FILE* fo = fopen(argv[3], "wb");
    if (!fo) return 4;
    fwrite(oh, sizeof(int), 5, fo);
    fwrite(raw_cc.data(), sizeof(float), n, fo);
    fwrite(cc.data(), sizeof(float), n, fo);
    fclose(fo);
    printf("{\"mode\": \"thick\", \"edges\": [%d, %d], \"thickness\": %d, \"offset_z\": %d, \"tile\": [%d, %d]}\n",
           oh[1], oh[2], oh[3], oh[4], calc.m_aiTileSize[0], calc.m_aiTileSize[1]);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc >= 2 && std::string(argv[1]) == "stack") return run_stack(argc, argv);
    if (argc >= 2 && std::string(argv[1]) == "thick") return run_thick(argc, argv);
    fprintf(stderr,
            "usage: %s stack in.bin params.bin out.bin seed bin size_axis\n"
            "       %s thick vol.bin out.bin bin\n",
            argv[0], argv[0]);
    return 2;
}
