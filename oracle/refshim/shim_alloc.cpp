/*
 * shim_alloc.cpp -- test infrastructure only; linked into oracle/_ref/clast_ref.
 *
 * With Thrust's CPP device system every thrust::device_vector is allocated
 * through the aligned global operator new.  The reference reads a few bytes
 * outside some of those vectors (the strided target k-mers near a window's
 * end in CDeviceHashTable.cu:37-55, and the DP's target bases before a
 * window's first sequence or past its last one in krnlAlignment.cu:121-128,
 * 234-241).  On a GPU those bytes are whatever lies next to the allocation.
 * Here every allocation gets 64 bytes of 'N' on both sides, so those reads
 * see a fixed non-ACGT base -- the same definition the oracle and the CUDA
 * kernels use for bases outside a window.
 */
#include <cstdlib>
#include <cstring>
#include <new>

namespace {
constexpr std::size_t kPad = 64;
std::size_t pad_for(std::size_t align) { return align > kPad ? align : kPad; }
void* padded_alloc(std::size_t n, std::size_t align) {
  const std::size_t pad = pad_for(align);
  const std::size_t total = ((pad + n + pad + align - 1) / align) * align;
  char* raw = static_cast<char*>(std::aligned_alloc(align < 16 ? 16 : align, total));
  if (!raw) throw std::bad_alloc();
  std::memset(raw, 'N', pad);
  std::memset(raw + pad + n, 'N', total - pad - n);
  return raw + pad;
}
void padded_free(void* p, std::size_t align) {
  if (p) std::free(static_cast<char*>(p) - pad_for(align));
}
}  // namespace

void* operator new(std::size_t n, std::align_val_t a) { return padded_alloc(n, static_cast<std::size_t>(a)); }
void* operator new[](std::size_t n, std::align_val_t a) { return padded_alloc(n, static_cast<std::size_t>(a)); }
void operator delete(void* p, std::align_val_t a) noexcept { padded_free(p, static_cast<std::size_t>(a)); }
void operator delete[](void* p, std::align_val_t a) noexcept { padded_free(p, static_cast<std::size_t>(a)); }
void operator delete(void* p, std::size_t, std::align_val_t a) noexcept { padded_free(p, static_cast<std::size_t>(a)); }
void operator delete[](void* p, std::size_t, std::align_val_t a) noexcept { padded_free(p, static_cast<std::size_t>(a)); }
