// Compatibility header: boost::math classification functions mapped to <cmath>.
#pragma once
#include <cmath>
namespace boost { namespace math { using std::isfinite; using std::fpclassify; using std::isnan; using std::isinf; } }
