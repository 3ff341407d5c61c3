// Test infrastructure only: writes a volume with the reference's own MRC
// writer (LibSrc/Mrcfile Mrc::CSaveMrc, compiled from the reference sources
// by oracle/ref/build_ref.sh into oracle/_ref/ref_mrc) in the sequence
// CAsyncSaveVol::mSaveVol uses (DataUtil/CAsyncSaveVol.cpp:97-118).  Parity
// target for the volume-file tests; nothing in the product links or calls it.
//
//   ref_mrc <in.bin> <out.mrc>
//     in.bin: int32 nx, ny, nz; float32 pixel size; float32 tilts[nz];
//             float32 frames[nz][ny][nx]
#include <cstdio>
#include <vector>

#include "Mrcfile/Include/CMrcFileInc.h"

static bool read_all(FILE* f, void* p, size_t n) { return fread(p, 1, n, f) == n; }

int main(int argc, char** argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s in.bin out.mrc\n", argv[0]);
        return 2;
    }
    FILE* fi = fopen(argv[1], "rb");
    if (!fi) return 3;
    int size[3];
    float pix = 0.f;
    if (!read_all(fi, size, sizeof(size)) || !read_all(fi, &pix, sizeof(pix))) return 3;
    const int nx = size[0], ny = size[1], nz = size[2];
    std::vector<float> tilts(nz);
    std::vector<float> frames((size_t)nx * ny * nz);
    if (!read_all(fi, tilts.data(), sizeof(float) * nz) || !read_all(fi, frames.data(), sizeof(float) * frames.size()))
        return 3;
    fclose(fi);
    Mrc::CSaveMrc save;
    if (!save.OpenFile(argv[2])) return 4;
    save.SetMode(Mrc::eMrcFloat);
    save.SetExtHeader(0, 32, 0);
    save.SetImgSize(size, size[2], 1, pix);
    save.m_pSaveMain->DoIt();
    for (int i = 0; i < nz; i++) {
        float tilt = tilts[i];
        save.m_pSaveExt->SetTilt(i, &tilt, 1);
        save.m_pSaveExt->DoIt();
        save.m_pSaveImg->DoIt(i, frames.data() + (size_t)i * nx * ny);
    }
    save.CloseFile();
    printf("{\"mode\": \"mrc\", \"size\": [%d, %d, %d]}\n", nx, ny, nz);
    return 0;
}
