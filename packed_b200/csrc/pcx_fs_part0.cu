// Variants of the one-launch four-step kernel, part 0 (see pcx_fs_launch.cuh).
#include "pcx_fs_launch.cuh"

PCX_FS_PART(pcx_fs_part0) {
    PCX_FS_VARIANT(float, 7, 6, 2, 3)
    PCX_FS_VARIANT(float, 6, 7, 2, 3)
    PCX_FS_VARIANT(float, 7, 7, 2, 3)
    PCX_FS_VARIANT(float, 7, 7, 1, 3)
    PCX_FS_VARIANT(float, 8, 7, 2, 3)
    PCX_FS_VARIANT(float, 7, 8, 2, 3)
    PCX_FS_VARIANT(float, 8, 8, 2, 3)
    PCX_FS_VARIANT(float, 9, 7, 2, 3)
    PCX_FS_VARIANT(float, 7, 9, 2, 3)
    return cudaErrorNotSupported;
}
