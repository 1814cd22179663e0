/* Umbrella header of the GPU phase-retrieval library (drop-in subset of the
 * reference's include/spimage.h for the phasing path). */
#ifndef SPB_SPIMAGE_H
#define SPB_SPIMAGE_H
#include "spimage/image.h"
#include "spimage/linear_alg.h"
#include "spimage/mem_util.h"
#include "spimage/list.h"
#include "spimage/map.h"
#include "spimage/image_util.h"
#include "spimage/fft.h"
#include "spimage/image_filter.h"
#include "spimage/support_update.h"
#include "spimage/phasing.h"
#include "spimage/prtf.h"
#endif
