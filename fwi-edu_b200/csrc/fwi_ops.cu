// fwi_ops.cu -- checkpoint-store bookkeeping of the reference interface.
#include <cmath>
#include "../../include/fwi_b200.h"
#include "fwi_setup.h"

// calculate_memory_cost_checkpoint, checkpoint.c:267-298: GB of the (nCheckPoint + d - 2)-frame store
extern "C" float calculate_memory_cost_checkpoint(int nt, int NX, int NZ)
{
    int d = fwi_ck_interval(nt), n = fwi_ck_count(nt);
    int ntPoint = n + d - 2;
    return 1.0f * (ntPoint * NZ * NX * (int)sizeof(float)) / powf(1024.0f, 3);
}
