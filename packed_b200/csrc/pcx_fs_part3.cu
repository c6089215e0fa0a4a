// Variants of the one-launch four-step kernel, part 3 (see pcx_fs_launch.cuh).
#include "pcx_fs_launch.cuh"

PCX_FS_PART(pcx_fs_part3) {
    PCX_FS_VARIANT(float, 9, 10, 1, 3)
    PCX_FS_VARIANT(float, 10, 10, 1, 2)
    PCX_FS_VARIANT(float, 10, 10, 1, 3)
    PCX_FS_VARIANT(double, 7, 7, 2, 3)
    PCX_FS_VARIANT(double, 8, 7, 2, 3)
    PCX_FS_VARIANT(float, 6, 8, 2, 3)
    PCX_FS_VARIANT(float, 6, 9, 2, 3)
    return cudaErrorNotSupported;
}
