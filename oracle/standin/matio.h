/* oracle/standin/matio.h -- TEST INFRASTRUCTURE (the oracle): declarations of
 * the matio (tbeu/matio) interface that the reference's
 * include/uncc_sar_matio.hpp and src/autofocus/cpu/autofocus_cpu.cpp name,
 * so that the latter compiles into oracle/_ref for its PGA routine.  matio is
 * not installed here; the functions are defined as failing stubs in
 * oracle/ref_pga_harness.cpp (the MAT reader of that file's main() is never
 * run).  Only names and signatures of the public interface are declared. */
#pragma once
#include <stddef.h>

enum mat_acc { MAT_ACC_RDONLY = 0, MAT_ACC_RDWR = 1 };
enum matio_classes {
    MAT_C_EMPTY = 0, MAT_C_CELL, MAT_C_STRUCT, MAT_C_OBJECT, MAT_C_CHAR, MAT_C_SPARSE, MAT_C_DOUBLE,
    MAT_C_SINGLE, MAT_C_INT8, MAT_C_UINT8, MAT_C_INT16, MAT_C_UINT16, MAT_C_INT32, MAT_C_UINT32,
    MAT_C_INT64, MAT_C_UINT64, MAT_C_FUNCTION, MAT_C_OPAQUE
};
enum matio_types {
    MAT_T_UNKNOWN = 0, MAT_T_INT8, MAT_T_UINT8, MAT_T_INT16, MAT_T_UINT16, MAT_T_INT32, MAT_T_UINT32,
    MAT_T_SINGLE, MAT_T_DOUBLE, MAT_T_INT64, MAT_T_UINT64, MAT_T_MATRIX, MAT_T_COMPRESSED, MAT_T_UTF8,
    MAT_T_UTF16, MAT_T_UTF32, MAT_T_STRING, MAT_T_CELL, MAT_T_STRUCT, MAT_T_ARRAY, MAT_T_FUNCTION
};
typedef struct mat_complex_split_t {
    void *Re;
    void *Im;
} mat_complex_split_t;
typedef struct matvar_t {
    size_t nbytes;
    int rank;
    enum matio_types data_type;
    int data_size;
    enum matio_classes class_type;
    int isComplex;
    int isGlobal;
    int isLogical;
    size_t *dims;
    char *name;
    void *data;
    int mem_conserve;
    int compression;
    void *internal;
} matvar_t;
typedef struct _mat_t mat_t;

#ifdef __cplusplus
extern "C" {
#endif
mat_t *Mat_Open(const char *matname, int mode);
int Mat_Close(mat_t *mat);
matvar_t *Mat_VarReadNext(mat_t *mat);
void Mat_VarFree(matvar_t *matvar);
unsigned Mat_VarGetNumberOfFields(matvar_t *matvar);
matvar_t *Mat_VarGetStructFieldByIndex(matvar_t *matvar, size_t field_index, size_t index);
void Mat_VarPrint(matvar_t *matvar, int printdata);
int Mat_VarReadDataAll(mat_t *mat, matvar_t *matvar);
#ifdef __cplusplus
}
#endif
