// shm.cpp -- Corr32 shared-memory image publisher.
//
// Same layout as the reference's Corr32 (src/rx_host_corr.cu:97-105) so its
// viewer (src/peek32.cpp:173-189) can read it: {u32 magic 0x43523343, w, h,
// nch; u64 write_seq} followed by img[nch][h][w], vmax[nch], vmin[nch];
// write_seq is stored with release ordering after each frame (:236).
#include <fcntl.h>
#include <sys/mman.h>
#include <unistd.h>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include "mixer.h"

struct mixer_shm {
    std::string name;
    void* base;
    size_t bytes;
    int32_t nch, G;
};

namespace {
struct Corr32Header {
    uint32_t magic, w, h, nch;
    uint64_t write_seq;
};
static_assert(sizeof(Corr32Header) == 24, "Corr32 header is 24 bytes");
}  // namespace

extern "C" int mixer_shm_open(const char* name, int32_t nch, int32_t G, mixer_shm** out) {
    if (!name || name[0] != '/' || nch <= 0 || G <= 0 || !out) return MIXER_EINVAL;
    *out = nullptr;
    const size_t bytes = sizeof(Corr32Header) + sizeof(float) * ((size_t)nch * G * G + 2 * (size_t)nch);
    shm_unlink(name);
    const int fd = shm_open(name, O_CREAT | O_RDWR, 0666);
    if (fd < 0) return MIXER_EINVAL;
    if (ftruncate(fd, (off_t)bytes) != 0) {
        close(fd);
        return MIXER_ENOMEM;
    }
    void* p = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
    close(fd);
    if (p == MAP_FAILED) return MIXER_ENOMEM;
    std::memset(p, 0, bytes);
    Corr32Header* h = static_cast<Corr32Header*>(p);
    h->magic = 0x43523343u;
    h->w = (uint32_t)G;
    h->h = (uint32_t)G;
    h->nch = (uint32_t)nch;
    mixer_shm* s = new mixer_shm{name, p, bytes, nch, G};
    *out = s;
    return MIXER_OK;
}

extern "C" int mixer_shm_publish(mixer_shm* s, const float* img, const float* vmax,
                                 const float* vmin, uint64_t write_seq) {
    if (!s || !img) return MIXER_EINVAL;
    uint8_t* base = static_cast<uint8_t*>(s->base);
    float* dimg = reinterpret_cast<float*>(base + sizeof(Corr32Header));
    const size_t npix = (size_t)s->nch * s->G * s->G;
    std::memcpy(dimg, img, npix * sizeof(float));
    if (vmax) std::memcpy(dimg + npix, vmax, (size_t)s->nch * sizeof(float));
    if (vmin) std::memcpy(dimg + npix + s->nch, vmin, (size_t)s->nch * sizeof(float));
    Corr32Header* h = reinterpret_cast<Corr32Header*>(base);
    __atomic_store_n(&h->write_seq, write_seq, __ATOMIC_RELEASE);
    return MIXER_OK;
}

extern "C" int mixer_shm_close(mixer_shm* s, int32_t unlink_name) {
    if (!s) return MIXER_OK;
    munmap(s->base, s->bytes);
    if (unlink_name) shm_unlink(s->name.c_str());
    delete s;
    return MIXER_OK;
}
