// The drop-in: AreTomo3's two reconstruction entry points with their bodies
// replaced by calls into libat3r (include/at3r.h).  This translation unit
// takes the place of AreTomo/Recon/CDoWbpRecon.cpp and CDoSartRecon.cpp in an
// AreTomo3 build; it compiles against the reference's own headers
// (AreTomo/Recon/CReconInc.h:238-306 declares both classes), so the classes,
// their callers (CAreTomoMain::mWbpRecon / mSartRecon, CCalcVolThick::DoIt,
// CAlignMetric::Calculate) and the object layout stay as they are.
//
// Kept from the reference (CDoWbpRecon.cpp:28-47, CDoSartRecon.cpp:30-57):
//   * the returned volume is a new CTiltSeries of {nx / 2 * 2, iVolZ, ny}
//     whose frame y is the XZ slice at y with z flipped, owned by the caller;
//   * the tilt series is read, not modified; the tilt angles are
//     CAlignParam::GetTilts(false);
//   * SART's relaxation is 1 / iNumSubsets and its fill table is seeded with
//     time(0) (at3r_geom_init's defaults).
// Changed: the reference aborts the process on a CUDA error
// (MaUtil/CSimpleFuncs.cpp:53-62); here DoIt prints the library's message and
// returns NULL.
//
// Build (AreTomo3 tree): add this file in place of the two .cpp files, add
// <repo>/include to the include path, link with -L<repo>/aretomo3_b200 -lat3r.
#include "AreTomo/Recon/CReconInc.h"
#include "AreTomo/MrcUtil/CMrcUtilInc.h"
#include "at3r.h"

#include <cstdio>

using namespace McAreTomo::AreTomo::Recon;

namespace {

// Runs one plan over the series' host frames into a new volume series.
MD::CTiltSeries* at3r_reconstruct(MD::CTiltSeries* ts, at3r_geom& g)
{
    int vol_size[3] = {ts->m_aiStkSize[0] / 2 * 2, g.vol_z, ts->m_aiStkSize[1]};
    MD::CTiltSeries* vol = new MD::CTiltSeries;
    vol->Create(vol_size);
    at3r_plan* plan = nullptr;
    at3r_status s = at3r_plan_create(&g, &plan);
    if (s == AT3R_OK)
        s = at3r_run_host(plan, reinterpret_cast<const float* const*>(ts->GetFrames()),
                          reinterpret_cast<float* const*>(vol->GetFrames()), nullptr);
    at3r_plan_destroy(plan);
    if (s != AT3R_OK) {
        fprintf(stderr, "at3r reconstruction failed: %s (%s)\n", at3r_status_str(s), at3r_last_error());
        delete vol;
        return nullptr;
    }
    return vol;
}

void fill_series(at3r_geom& g, MD::CTiltSeries* ts, MAM::CAlignParam* aln, int iVolZ)
{
    g.nx = ts->m_aiStkSize[0];
    g.ny = ts->m_aiStkSize[1];
    g.n_tilts = ts->m_aiStkSize[2];
    g.vol_z = iVolZ;
    g.tilts_deg = aln->GetTilts(false);
}

}  // namespace

CDoWbpRecon::CDoWbpRecon(void) { m_pVolSeries = 0L; }

CDoWbpRecon::~CDoWbpRecon(void) { this->Clean(); }

void CDoWbpRecon::Clean(void)
{
    CDoBaseRecon::Clean();
    m_aTomoWbp.Clean();
    if (m_pVolSeries != 0L) delete m_pVolSeries;
    m_pVolSeries = 0L;
}

MD::CTiltSeries* CDoWbpRecon::DoIt(MD::CTiltSeries* pTiltSeries, MAM::CAlignParam* pAlignParam, int iVolZ)
{
    m_pTiltSeries = pTiltSeries;
    m_pAlignParam = pAlignParam;
    m_iVolZ = iVolZ;
    at3r_geom g;
    at3r_geom_init(&g, AT3R_WBP);
    fill_series(g, pTiltSeries, pAlignParam, iVolZ);
    return at3r_reconstruct(pTiltSeries, g);
}

CDoSartRecon::CDoSartRecon(void)
{
    m_iNumIters = 1;
    m_iNumSubsets = 1;
    m_pVolSeries = 0L;
}

CDoSartRecon::~CDoSartRecon(void) { this->Clean(); }

void CDoSartRecon::Clean(void)
{
    CDoBaseRecon::Clean();
    m_aTomoSart.Clean();
    if (m_pVolSeries != 0L) delete m_pVolSeries;
    m_pVolSeries = 0L;
}

MD::CTiltSeries* CDoSartRecon::DoIt(MD::CTiltSeries* pTiltSeries, MAM::CAlignParam* pAlignParam, int iStartTilt,
                                    int iNumTilts, int iVolZ, int iIterations, int iNumSubsets)
{
    m_pTiltSeries = pTiltSeries;
    m_pAlignParam = pAlignParam;
    m_iVolZ = iVolZ;
    m_iStartTilt = iStartTilt;
    m_iNumTilts = iNumTilts;
    m_iNumIters = iIterations;
    m_iNumSubsets = iNumSubsets;
    at3r_geom g;
    at3r_geom_init(&g, AT3R_SART);
    fill_series(g, pTiltSeries, pAlignParam, iVolZ);
    g.start_tilt = iStartTilt;
    g.num_tilts = iNumTilts;
    g.iterations = iIterations;
    g.subsets = iNumSubsets;
    return at3r_reconstruct(pTiltSeries, g);
}
