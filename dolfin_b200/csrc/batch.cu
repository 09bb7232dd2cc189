// batch.cu -- batched multi-mesh assembly (placeholder until the persistent kernel lands).
#include "internal.h"
extern "C" {
int db2_batch_create(int, const db2_pattern*, const db2_form*, const double* const*, double* const*,
                     int, int, int, db2_batch*) { return DB2_ERR_UNSUPPORTED; }
int db2_batch_info(db2_batch, int64_t*, int64_t*, int*) { return DB2_ERR_UNSUPPORTED; }
int db2_batch_assemble(db2_batch, int, void*) { return DB2_ERR_UNSUPPORTED; }
int db2_batch_assemble_loop(db2_batch, int, void*) { return DB2_ERR_UNSUPPORTED; }
int db2_batch_destroy(db2_batch) { return DB2_OK; }
}
