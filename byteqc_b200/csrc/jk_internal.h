// Internal helpers of jk_host.cu shared with other translation units of
// libjk.so (not part of the C-ABI).
#pragma once
#include "jk_common.cuh"
#include "../../include/byteqc_jk.h"

int jk_internal_set_err(int code, const char* msg);
// pair counts of the two classes and the working-basis size
int jk_internal_class_info(const jk_basis_t* b, int cp_ij, int cp_kl, int* n_ij, int* n_kl, int* nao);
void jk_internal_fill_seg(const jk_basis_t* b, int cp_ij, int cp_kl, const long long* qoff, int n_ij,
                          const double* dm, int n_dm, double* vj, double* vk, JKSeg* out);
// launch the class kernel of (cp_ij, cp_kl) on a device segment table of one entry
int jk_internal_launch(const jk_basis_t* b, int cp_ij, int cp_kl, const JKSeg& seg, const long long* d_task0,
                       long long max_tasks, void* stream);
