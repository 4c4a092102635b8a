/* Source-compatibility entry for code written against the reference's
 * include/physis/physis.h with PHYSIS_CUDA defined (what the CUDA target's
 * generated .cuda.cu files include): everything it needs is declared by the
 * B200 runtime's C ABI. */
#ifndef PHYSIS_B200_COMPAT_PHYSIS_H_
#define PHYSIS_B200_COMPAT_PHYSIS_H_
#include "../physis_b200.h"
#endif
