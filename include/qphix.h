/*
 * qphix.h -- umbrella header of the QPhiX C API served by libqphix_b200.so.
 * Replaces the reference qphix.h: the same QPHIX_Precision /
 * QPHIX_PrecisionInt selection logic (default single precision), then the
 * precision-independent and the F3/D3 headers.
 */
#ifndef _QPHIX_H
#define _QPHIX_H

#ifndef QPHIX_Precision
#  ifndef QPHIX_PrecisionInt
#    define QPHIX_PrecisionInt 1
#  endif
#  if QPHIX_PrecisionInt == 1
#    define QPHIX_Precision 'F'
#    define QPHIX_PrecisionLetter F
#  elif QPHIX_PrecisionInt == 2
#    define QPHIX_Precision 'D'
#    define QPHIX_PrecisionLetter D
#  else
#    error "bad QPHIX_PrecisionInt"
#  endif
#else
#  ifndef QPHIX_PrecisionInt
#    if QPHIX_Precision == 'F'
#      define QPHIX_PrecisionInt 1
#      define QPHIX_PrecisionLetter F
#    elif QPHIX_Precision == 'D'
#      define QPHIX_PrecisionInt 2
#      define QPHIX_PrecisionLetter D
#    else
#      error "bad QPHIX_Precision"
#    endif
#  else
#    if QPHIX_Precision == 'F'
#      if QPHIX_PrecisionInt != 1
#        error "inconsistent QPHIX_Precision='F' and QPHIX_PrecisionInt"
#      endif
#      define QPHIX_PrecisionLetter F
#    elif QPHIX_Precision == 'D'
#      if QPHIX_PrecisionInt != 2
#        error "inconsistent QPHIX_Precision='D' and QPHIX_PrecisionInt"
#      endif
#      define QPHIX_PrecisionLetter D
#    else
#      error "bad QPHIX_Precision"
#    endif
#  endif
#endif

#include <qphix_int.h>
#include <qphix_f3.h>
#include <qphix_d3.h>
#endif
