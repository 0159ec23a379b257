// Compatibility header: boost::chrono mapped to std::chrono (used only by the reference's timers).
#pragma once
#include <chrono>
#include <ratio>
namespace boost { namespace chrono = std::chrono; using std::nano; using std::micro; using std::milli; }
