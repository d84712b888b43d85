// Generated d classes 0..9: (ds|ss) .. (dp|ds).
#define HLC_FIRST 0
#define HLC_LAST 9
#define HLC_PART_LAUNCH hlc_part_a_launch
#define HLC_PART_INIT hlc_part_a_init
#include "hlc_part.cuh"
