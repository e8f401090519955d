// Device status bits written by libjlcgpu kernels into the context's status word.
#pragma once

#define JLC_DEV_TIMEOUT 0x1   // a bounded mbarrier/flag wait expired
#define JLC_DEV_BADARG 0x2    // a kernel saw an argument it cannot handle
#define JLC_DEV_NONFINITE 0x4 // Ozaki split met Inf/NaN (handled by the FP64 route)
