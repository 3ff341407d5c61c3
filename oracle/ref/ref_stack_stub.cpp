// Test infrastructure only.  The reference's CCalcVolThick.cpp and
// CCorrectUtil.cpp name classes whose code the input-stage driver never
// reaches (the full CCorrTomoStack pipeline object, the temporary-file
// writers, the local cross-correlation of mMeasure, real-space binning).
// These empty definitions satisfy the linker; each one aborts if called.
#include "AreTomo/Recon/CReconInc.h"
#include "AreTomo/Correct/CCorrectInc.h"
#include "CMcAreTomoInc.h"
#include <cstdio>
#include <cstdlib>

static void never(const char* what)
{
    fprintf(stderr, "ref_stack: unexpected call to %s\n", what);
    abort();
}

namespace McAreTomo {
CInput* CInput::GetInstance(void) { never("CInput::GetInstance"); return nullptr; }
namespace MaUtil {
CSaveTempMrc::CSaveTempMrc(void) {}
CSaveTempMrc::~CSaveTempMrc(void) {}
void CSaveTempMrc::SetFile(char*, const char*) { never("CSaveTempMrc::SetFile"); }
void CSaveTempMrc::DoMany(void**, int, int*) { never("CSaveTempMrc::DoMany"); }
}  // namespace MaUtil
namespace AreTomo {
namespace Util {
GLocalCC2D::GLocalCC2D(void) {}
GLocalCC2D::~GLocalCC2D(void) {}
void GLocalCC2D::SetSizes(int*, int*) {}
float GLocalCC2D::DoIt(float*, float*, int*) { never("GLocalCC2D::DoIt"); return 0.f; }
GBinImage2D::GBinImage2D(void) {}
GBinImage2D::~GBinImage2D(void) {}
void GBinImage2D::GetBinSize(int*, bool, int, int*, bool) { never("GBinImage2D::GetBinSize"); }
}  // namespace Util
namespace Correct {
CFourierCropImage::CFourierCropImage(void) {}
CFourierCropImage::~CFourierCropImage(void) {}
CCorrTomoStack::CCorrTomoStack(void) { never("CCorrTomoStack"); }
CCorrTomoStack::~CCorrTomoStack(void) {}
void CCorrTomoStack::Set0(int) {}
void CCorrTomoStack::Set1(int, float) {}
void CCorrTomoStack::Set2(float, bool, bool) {}
void CCorrTomoStack::Set3(bool, bool, bool) {}
void CCorrTomoStack::Set4(bool) {}
void CCorrTomoStack::DoIt(int, MrcUtil::CAlignParam*) {}
DataUtil::CTiltSeries* CCorrTomoStack::GetCorrectedStack(bool) { return nullptr; }
}  // namespace Correct
}  // namespace AreTomo
}  // namespace McAreTomo
