// TEST INFRASTRUCTURE ONLY -- part of the owl::common stand-in (the box and
// vector types live in owl-common.h; nothing else of this header is used by
// the compiled reference files).
#pragma once
#include "owl/common/owl-common.h"
