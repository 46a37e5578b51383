/* so3.h -- umbrella header of the drop-in SO3 C ABI (reference include/so3/so3.h). */
#ifndef SO3
#define SO3
#include "so3_types.h"
#include "so3_error.h"
#include "so3_sampling.h"
#include "so3_core.h"
#include "so3_conv.h"
#include "so3_adjoint.h"
#endif
