/* Minimal stand-in for the MKL type header, used only to compile the
 * reference (bem3_emf_qd2) as a CPU oracle where MKL is not installed.
 * ILP64 integer width matches the reference build flag -DMKL_ILP64. */
#ifndef ORACLE_MKL_TYPES_STUB_H
#define ORACLE_MKL_TYPES_STUB_H
typedef long long MKL_INT;
typedef struct { double real, imag; } MKL_Complex16;
typedef struct { float real, imag; } MKL_Complex8;
#endif
