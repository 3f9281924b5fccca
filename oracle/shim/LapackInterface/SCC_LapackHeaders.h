// Stand-in for SCC_LapackHeaders.h (see SCC_LapackMatrix.h). It leaves EXTERNAL_LAPACK undefined, so
// the reference's Dstebz_C (Dstebz_C.h:12-16) uses its own translation of dstebz, as the CPU build
// with RC_WITHOUT_LAPACK_ does.
#pragma once
