// gd_tune.cpp -- process-wide launch tuning knobs.
//
// No counterpart in the reference (its launch shapes are compile-time
// constants).  Each knob selects among kernel variants compiled into the
// library or sets a launch shape; 0 always means the built-in default.  The
// autotuner (compression_b200/autotune.py) times the choices on the device
// and sets the fastest.
#include <atomic>

#include "../../../include/gd.h"

namespace {
std::atomic<int> g_knob[GD_TUNE_COUNT];
}

extern "C" int gd_tune_set(int key, int value) {
    if (key < 0 || key >= GD_TUNE_COUNT || value < 0) return -1;
    return g_knob[key].exchange(value);
}

extern "C" int gd_tune_get(int key) {
    if (key < 0 || key >= GD_TUNE_COUNT) return -1;
    return g_knob[key].load();
}
