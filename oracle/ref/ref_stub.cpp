// Test infrastructure only.  CDarkFrames (compiled in because CAlignParam's
// translation unit pulls it into the link) names CTsPackage, which is never
// reached on the Recon path.  These two definitions satisfy the linker.
#include "DataUtil/CDataUtilInc.h"

namespace McAreTomo { namespace DataUtil {
CTsPackage* CTsPackage::GetInstance(int) { return nullptr; }
CTiltSeries* CTsPackage::GetSeries(int) { return nullptr; }
} }
