// Generated d classes 13..13: (dd|dp).
#define HLC_FIRST 13
#define HLC_LAST 13
#define HLC_PART_LAUNCH hlc_part_c_launch
#define HLC_PART_INIT hlc_part_c_init
#include "hlc_part.cuh"
