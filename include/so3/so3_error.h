/*
 * so3_error.h -- error convention of the drop-in (reference
 * include/so3/so3_error.h:19-33): invalid parameters print a message and
 * terminate the process.  libso3gpu additionally records a status and message
 * for every call (so3gpu_last_status / so3gpu_last_error in so3gpu.h) and can
 * be switched to return instead of exit (so3gpu_set_error_mode).
 */
#ifndef SO3_ERROR
#define SO3_ERROR

#include <stdio.h>
#include <stdlib.h>

#define SO3_ERROR_GENERIC(comment)                                                       \
  {                                                                                      \
    printf("ERROR: %s.\n", comment);                                                     \
    printf("ERROR: %s <%s> %s %s %s %d.\n", "Occurred in function", __func__, "of file", \
           __FILE__, "on line", __LINE__);                                               \
    exit(1);                                                                             \
  }

#define SO3_ERROR_MEM_ALLOC_CHECK(pointer)                                               \
  if (pointer == NULL) {                                                                 \
    SO3_ERROR_GENERIC("Memory allocation failed")                                        \
  }

#endif
