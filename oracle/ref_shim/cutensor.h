/* Stand-in for the legacy cuTENSOR 1.x header, which is not installed here.
 * The reference's collision table builders (getOmega.cu, getFcL.cu) include
 * it only through setup.hpp, for the status type of an error-printing helper
 * (setup.cpp); they call no cuTENSOR function.  Declares that type alone, so
 * those sources compile unmodified into oracle/_ref.  Test infrastructure. */
#ifndef HP_REF_SHIM_CUTENSOR_H
#define HP_REF_SHIM_CUTENSOR_H
typedef enum { CUTENSOR_STATUS_SUCCESS = 0 } cutensorStatus_t;
#endif
