/* thread.h of the exafmm-beta include tree, for drivers written against it: the
 * B200 engine's C++ facade provides its classes (exafmm_b200.hpp). */
#ifndef EXAFMM_COMPAT_THREAD_H
#define EXAFMM_COMPAT_THREAD_H
#include "../exafmm_b200.hpp"
#endif
