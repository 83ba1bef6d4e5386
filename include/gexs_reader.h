/*
 * gexs_reader.h — flat C view of B200ExomolReader (gexs_b200/host), the
 * StateReader drop-in beside the reference's ExomolStateReader
 * (Readers/Exomol/ExomolStateReader.h:30-48; interface Readers/StateReader.h):
 * constructor -> gexs_reader_create, OpenFile -> gexs_reader_open,
 * ReadNextState (6 arguments) -> gexs_reader_next, ComputePartition ->
 * gexs_reader_partition, CloseFile -> gexs_reader_close.  Parsing runs on
 * the GPU (see the ExoMol ingest section of gexs_b200.h); records stream in
 * file order unless sort_by_nu.  Every function returns a GEXS_* status.
 */
#ifndef GEXS_READER_H
#define GEXS_READER_H

#include <stdint.h>
#include "gexs_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gexs_reader gexs_reader;

/* broad_path may be NULL or name a missing file (then: defaults) */
int gexs_reader_create(const char* states_path, const char* broad_path, double default_gamma,
                       double default_n, int device, int broad_mode, int sort_by_nu,
                       gexs_reader** out);
int gexs_reader_open(gexs_reader* r, const char* trans_path, int64_t* ntrans);
/* *more = 0 after the last record (ExomolStateReader::ReadNextState false) */
int gexs_reader_next(gexs_reader* r, double* nu, double* gns, double* e_i, double* aif,
                     double* gam, double* n, int* more);
int gexs_reader_partition(gexs_reader* r, double temperature, double* q);
/* the open file's lines in device memory (valid until close/destroy) */
int gexs_reader_device_lines(gexs_reader* r, gexs_lines* out);
int gexs_reader_close(gexs_reader* r);
int gexs_reader_destroy(gexs_reader* r);

#ifdef __cplusplus
}
#endif

#endif
