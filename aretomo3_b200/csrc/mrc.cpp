// C-ABI implementation of the volume file (at3r_mrc_write): the MRC file
// DataUtil/CAsyncSaveVol.cpp:82-126 writes through LibSrc/Mrcfile's CSaveMrc.
#include "at3r.h"
#include "at3r_internal.h"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

at3r_status mrc_err(at3r_status s, const std::string& msg)
{
    at3r_set_last_error(msg.c_str());
    return s;
}

template <typename T>
void put(unsigned char* h, size_t off, T v)
{
    std::memcpy(h + off, &v, sizeof(T));
}

// The 1024-byte main header CSaveMainHeader writes for a float volume
// (Header/CSaveMainHeader.cpp: mSetDefault, SetImgSize, SetMode; the field
// offsets of CMainHeader, Include/CMrcFileInc.h).  Min / max / mean stay 0
// and there is no extended header: CAsyncSaveVol never sets the statistics,
// and CSaveMrc::SetImgSize resets the extended header it asked for before.
void mrc_header(unsigned char* h, int nx, int ny, int nz, float pix)
{
    std::memset(h, 0, 1024);
    put<int32_t>(h, 0, nx);
    put<int32_t>(h, 4, ny);
    put<int32_t>(h, 8, nz);
    put<int32_t>(h, 12, 2);                      // mode: 32-bit float
    put<int32_t>(h, 28, nx);                     // mx, my, mz: the sampling
    put<int32_t>(h, 32, ny);
    put<int32_t>(h, 36, nz);
    put<float>(h, 40, (float)nx * pix);          // cell lengths
    put<float>(h, 44, (float)ny * pix);
    put<float>(h, 48, (float)nz * pix);
    put<float>(h, 52, 90.f);                     // cell angles
    put<float>(h, 56, 90.f);
    put<float>(h, 60, 90.f);
    put<int32_t>(h, 64, 1);                      // mapc, mapr, maps
    put<int32_t>(h, 68, 2);
    put<int32_t>(h, 72, 3);
    put<int16_t>(h, 96, (int16_t)-16224);        // dvid
    std::memcpy(h + 104, "AGAR", 4);             // extended-header type
    put<int32_t>(h, 108, 2014 * 10);             // version
    put<int16_t>(h, 132, 1);                     // sub
    put<int16_t>(h, 160, 5);                     // type
    put<float>(h, 184, 90.f);                    // xtilt, ytilt, ztilt
    put<float>(h, 188, 90.f);
    put<float>(h, 192, 90.f);
    std::memcpy(h + 208, "MAP", 4);              // word 53 ("MAP" and its terminator)
    const uint32_t probe = 0x0a0b0c0du;
    unsigned char b0;
    std::memcpy(&b0, &probe, 1);
    const unsigned char stamp[4] = {b0 == 0x0a ? (unsigned char)0x11 : (unsigned char)0x44,
                                    b0 == 0x0a ? (unsigned char)0x11 : (unsigned char)0x44, 0, 0};
    std::memcpy(h + 212, stamp, 4);              // word 54: machine stamp
}

bool pwrite_all(int fd, const void* buf, size_t bytes, off_t off)
{
    const char* p = static_cast<const char*>(buf);
    while (bytes > 0) {
        const ssize_t w = pwrite(fd, p, std::min<size_t>(bytes, (size_t)1 << 30), off);
        if (w < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        if (w == 0) return false;
        p += w;
        off += w;
        bytes -= (size_t)w;
    }
    return true;
}

}  // namespace

extern "C" {

at3r_status at3r_mrc_write(const char* path, const float* const* frames, int nx, int ny, int nz, float pix_size)
{
    if (!path || !frames) return mrc_err(AT3R_ERR_INVALID_ARGUMENT, "null argument");
    if (nx < 1 || ny < 1 || nz < 1) return mrc_err(AT3R_ERR_INVALID_ARGUMENT, "sizes must be >= 1");
    for (int z = 0; z < nz; z++)
        if (!frames[z]) return mrc_err(AT3R_ERR_INVALID_ARGUMENT, "null frame pointer");
    const int fd = open(path, O_RDWR | O_CREAT | O_TRUNC, S_IRUSR | S_IWUSR | S_IWGRP | S_IRGRP | S_IROTH);
    if (fd < 0) return mrc_err(AT3R_ERR_IO, std::string("cannot open ") + path + ": " + std::strerror(errno));
    unsigned char header[1024];
    mrc_header(header, nx, ny, nz, pix_size);
    bool ok = pwrite_all(fd, header, sizeof(header), 0);
    int err = ok ? 0 : errno;
    // frames at 1024 + z * frame bytes, split over up to four writer threads;
    // each thread keeps the errno of its own failed write (errno is per thread)
    const size_t fbytes = (size_t)nx * ny * sizeof(float);
    const int nt = (int)std::max(1, std::min(4, nz));
    std::vector<int> errt(nt, 0);
    auto run = [&](int k, int stride) {
        for (int z = k; z < nz && !errt[k]; z += stride)
            if (!pwrite_all(fd, frames[z], fbytes, (off_t)(1024 + (size_t)z * fbytes))) errt[k] = errno ? errno : EIO;
    };
    if (ok) {
        std::vector<std::thread> th;
        try {
            for (int k = 1; k < nt; k++) th.emplace_back(run, k, nt);
        } catch (const std::exception&) {
            // no threads to be had: the frames the missing threads would have
            // written are written here, after the calling thread's own share
        }
        const int started = 1 + (int)th.size();
        run(0, nt);
        for (int k = started; k < nt; k++) run(k, nt);
        for (std::thread& t : th) t.join();
        for (int e : errt)
            if (e && ok) { ok = false; err = e; }
    }
    if (close(fd) != 0 && ok) { ok = false; err = errno; }
    if (!ok) return mrc_err(AT3R_ERR_IO, std::string("write to ") + path + " failed: " + std::strerror(err));
    return AT3R_OK;
}

}  // extern "C"
