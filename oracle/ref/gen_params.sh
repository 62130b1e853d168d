#!/bin/sh
# Writes a params header for one reference build configuration.  It defines
# PARAMS_H first, so the reference's own params.h (included by every file) is
# skipped and these values are used instead; the macro names and meanings are
# those of the reference's params.h.
# usage: gen_params.sh GPUNUMDIM NUMINDEXEDDIM DTYPE > params_override.h
cat <<H
#ifndef PARAMS_H
#define PARAMS_H
#include <omp.h>
#define GPUNUMDIM $1
#define NUMINDEXEDDIM $2
#define BLOCKSIZE 256
#define GPUSTREAMS 3
#define CPU_THREADS (omp_get_num_procs())
#define CPU_BATCH_SIZE 1024
#define DTYPE $3
#define REAL $3
#define MINLEN 32
#define STATIC_SPLIT_QUERIES 1
#define SILENT_GPU 1
#define COUNT_CANDIDATES 0
#define COUNT_CANDIDATES_GPU 0
#define COMPARE_CANDIDATES 0
#define NB_ARGS_MAX 6
#define FILENAME_ARG 1
#define EPSILON_ARG 2
#define DIM_ARG 3
#define SEARCHMODE_ARG 4
#define STATIC_PART_ARG 5
#define SM_GPU 0
#define SM_HYBRID 1
#define SM_HYBRID_STATIC 2
#define SM_CPU 3
#define SORT_BY_WORKLOAD 1
#endif
H
