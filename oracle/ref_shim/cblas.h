/* Minimal CBLAS prototype header used only to compile the reference's
 * dimension-tree sources (dimtree/ddttensor.hpp, dimtree/dimtrees.hpp) against
 * the OpenBLAS shared library that ships in this image. Test infrastructure. */
#ifndef ORACLE_REF_SHIM_CBLAS_H_
#define ORACLE_REF_SHIM_CBLAS_H_
#ifdef __cplusplus
extern "C" {
#endif
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef CBLAS_LAYOUT CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
void cblas_dgemm(CBLAS_LAYOUT, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int,
                 double, const double*, int, const double*, int, double, double*, int);
void cblas_dgemv(CBLAS_LAYOUT, CBLAS_TRANSPOSE, int, int, double, const double*, int,
                 const double*, int, double, double*, int);
void cblas_dcopy(int, const double*, int, double*, int);
double cblas_ddot(int, const double*, int, const double*, int);
double cblas_dnrm2(int, const double*, int);
void cblas_dscal(int, double, double*, int);
void cblas_dsyrk(CBLAS_LAYOUT, CBLAS_UPLO, CBLAS_TRANSPOSE, int, int, double,
                 const double*, int, double, double*, int);
void cblas_dsymv(CBLAS_LAYOUT, CBLAS_UPLO, int, double, const double*, int,
                 const double*, int, double, double*, int);
#ifdef __cplusplus
}
#endif
#endif
