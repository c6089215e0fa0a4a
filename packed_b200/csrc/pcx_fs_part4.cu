// Variants of the one-launch four-step kernel, part 4 (see pcx_fs_launch.cuh).
#include "pcx_fs_launch.cuh"

PCX_FS_PART(pcx_fs_part4) {
    PCX_FS_VARIANT(double, 8, 8, 2, 3)
    PCX_FS_VARIANT(double, 9, 8, 2, 3)
    PCX_FS_VARIANT(double, 9, 9, 2, 3)
    PCX_FS_VARIANT(double, 10, 9, 1, 2)
    PCX_FS_VARIANT(double, 10, 10, 1, 2)
    PCX_FS_VARIANT(float, 6, 10, 1, 3)
    PCX_FS_VARIANT(float, 7, 10, 1, 3)
    return cudaErrorNotSupported;
}
