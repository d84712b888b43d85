// Generated d classes 14..14: (dd|dd).
#define HLC_FIRST 14
#define HLC_LAST 14
#define HLC_PART_LAUNCH hlc_part_d_launch
#define HLC_PART_INIT hlc_part_d_init
#include "hlc_part.cuh"
