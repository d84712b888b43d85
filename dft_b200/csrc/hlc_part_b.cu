// Generated d classes 10..12: (dp|dp), (dd|pp), (dd|ds).
#define HLC_FIRST 10
#define HLC_LAST 12
#define HLC_PART_LAUNCH hlc_part_b_launch
#define HLC_PART_INIT hlc_part_b_init
#include "hlc_part.cuh"
