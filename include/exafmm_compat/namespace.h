/* namespace.h of the exafmm-beta include tree: EXAFMM_NAMESPACE names the
 * facade's namespace (exafmm_laplace; the engine is Laplace only). */
#ifndef EXAFMM_COMPAT_NAMESPACE_H
#define EXAFMM_COMPAT_NAMESPACE_H
#include "../exafmm_b200.hpp"
#endif
