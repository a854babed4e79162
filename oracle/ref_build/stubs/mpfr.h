/* Type-only MPFR declarations.  The reference's transforms.c pulls in its MPFR
 * connection-matrix code unconditionally; the oracle build only needs it to
 * compile and link.  The struct layout here is NOT the real one, so no MPFR
 * function may ever be called through this build. */
#ifndef ORACLE_STUB_MPFR_H
#define ORACLE_STUB_MPFR_H
typedef long mpfr_prec_t;
typedef int mpfr_sign_t;
typedef long mpfr_exp_t;
typedef enum {MPFR_RNDN = 0, MPFR_RNDZ, MPFR_RNDU, MPFR_RNDD, MPFR_RNDA} mpfr_rnd_t;
typedef struct {mpfr_prec_t p; mpfr_sign_t s; mpfr_exp_t e; void * d;} oracle_stub_mpfr_struct;
typedef oracle_stub_mpfr_struct mpfr_t[1];
typedef oracle_stub_mpfr_struct * mpfr_ptr;
typedef const oracle_stub_mpfr_struct * mpfr_srcptr;
void mpfr_init2(mpfr_ptr, mpfr_prec_t);
void mpfr_clear(mpfr_ptr);
int mpfr_set(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_set_d(mpfr_ptr, double, mpfr_rnd_t);
void mpfr_set_zero(mpfr_ptr, int);
int mpfr_add(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_sub(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_mul(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_div(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_add_d(mpfr_ptr, mpfr_srcptr, double, mpfr_rnd_t);
int mpfr_sub_d(mpfr_ptr, mpfr_srcptr, double, mpfr_rnd_t);
int mpfr_mul_d(mpfr_ptr, mpfr_srcptr, double, mpfr_rnd_t);
int mpfr_div_d(mpfr_ptr, mpfr_srcptr, double, mpfr_rnd_t);
int mpfr_d_div(mpfr_ptr, double, mpfr_srcptr, mpfr_rnd_t);
int mpfr_fma(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_fms(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_neg(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_sqrt(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_sqrt_ui(mpfr_ptr, unsigned long, mpfr_rnd_t);
int mpfr_rec_sqrt(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_gamma(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_ui_pow(mpfr_ptr, unsigned long, mpfr_srcptr, mpfr_rnd_t);
#endif
