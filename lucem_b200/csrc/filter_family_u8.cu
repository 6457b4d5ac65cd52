// filter_family_u8.cu -- the Gaussian-family tile kernels for uint8_t input
// (filter_family.cuh), in a translation unit of their own.
#include "filter_family.cuh"

namespace lucem {
namespace famk {

int planes_u8(const FamParams &p, void *stream) { return planes_t<uint8_t>(p, stream); }

int batch_u8(const FamParams &p, const FamImage *items_dev, int32_t n_items, int32_t n_tiles, void *stream) {
    return batch_t<uint8_t>(p, items_dev, n_items, n_tiles, stream);
}

int work_u8(const FamParams &p, const FamWork *work_dev, int32_t n_work, int32_t n_tiles_total, int32_t tile_base,
               int32_t *counter_dev, int32_t persistent_ctas, void *stream) {
    return work_t<uint8_t>(p, work_dev, n_work, n_tiles_total, tile_base, counter_dev, persistent_ctas, stream);
}

}  // namespace famk
}  // namespace lucem
