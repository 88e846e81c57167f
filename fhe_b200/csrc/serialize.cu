// A wire format for engine objects (keys, ciphertexts, plaintexts).  The reference
// declares a Data::write and a Bytearray (data/data.h:66, data/bytearray.h) with a
// DATA_VERSION of 5 but defines no format; this one is self-describing and checks
// the engine it is read into.  Little-endian, 8-byte aligned:
//
//   offset  field
//   0       magic "FHEB200D"
//   8       u32 format version (1), u32 reference data version (5)
//   16      u32 log N, u32 prime count, u32 chain count, u32 special prime count
//   32      u64 FNV-1a hash of the prime chain
//   40      i32 type, i32 flag, i32 moduli id, i32 polynomials, i32 limbs, i32 delta
//   64      f64 scale (high part), f64 scale - high part (the long double's rest)
//   80      polys x limbs x N int64 words, [poly][limb][N]
#include <cstring>

#include "engine.hpp"

namespace fhe_b200 {

namespace {

constexpr char kMagic[8] = {'F', 'H', 'E', 'B', '2', '0', '0', 'D'};
constexpr uint32_t kFormatVersion = 1;
constexpr uint32_t kReferenceDataVersion = 5;  // DATA_VERSION, data/version.h
constexpr size_t kHeaderBytes = 80;

uint64_t chain_hash(const Parameters &p) {
  uint64_t h = 1469598103934665603ULL;
  for (uint64_t q : p.q)
    for (int b = 0; b < 8; b++) {
      h ^= (q >> (8 * b)) & 0xFF;
      h *= 1099511628211ULL;
    }
  return h;
}

template <class T>
void put(uint8_t *buf, size_t off, T v) {
  std::memcpy(buf + off, &v, sizeof(T));
}

template <class T>
T get(const uint8_t *buf, size_t off) {
  T v;
  std::memcpy(&v, buf + off, sizeof(T));
  return v;
}

}  // namespace

size_t Engine::serialized_size(const Data &d) const {
  return kHeaderBytes + d.words() * sizeof(int64_t);
}

void Engine::serialize(const Data &d, void *buffer, size_t capacity) {
  const size_t size = serialized_size(d);
  if (!buffer || capacity < size)
    throw std::invalid_argument("serialize: the buffer is smaller than the serialized object.");
  uint8_t *b = static_cast<uint8_t *>(buffer);
  std::memset(b, 0, kHeaderBytes);
  std::memcpy(b, kMagic, sizeof(kMagic));
  put<uint32_t>(b, 8, kFormatVersion);
  put<uint32_t>(b, 12, kReferenceDataVersion);
  put<uint32_t>(b, 16, static_cast<uint32_t>(params.log_n));
  put<uint32_t>(b, 20, static_cast<uint32_t>(params.prime_count));
  put<uint32_t>(b, 24, static_cast<uint32_t>(params.chain_count));
  put<uint32_t>(b, 28, static_cast<uint32_t>(params.special_prime_count));
  put<uint64_t>(b, 32, chain_hash(params));
  put<int32_t>(b, 40, d.type);
  put<int32_t>(b, 44, d.flag);
  put<int32_t>(b, 48, d.moduli_id);
  put<int32_t>(b, 52, d.polys);
  put<int32_t>(b, 56, d.chains);
  put<int32_t>(b, 60, d.delta);
  const double hi = static_cast<double>(d.scale);
  put<double>(b, 64, hi);
  put<double>(b, 72, static_cast<double>(d.scale - static_cast<long double>(hi)));
  download(d, reinterpret_cast<int64_t *>(b + kHeaderBytes));
}

std::unique_ptr<Data> Engine::deserialize(const void *buffer, size_t size) {
  const std::string fn = "deserialize";
  if (!buffer || size < kHeaderBytes)
    throw std::invalid_argument(fn + ": the buffer is shorter than the header.");
  const uint8_t *b = static_cast<const uint8_t *>(buffer);
  if (std::memcmp(b, kMagic, sizeof(kMagic)) != 0)
    throw std::invalid_argument(fn + ": not a serialized engine object.");
  if (get<uint32_t>(b, 8) != kFormatVersion)
    throw std::invalid_argument(fn + ": unsupported format version.");
  if (get<uint32_t>(b, 16) != static_cast<uint32_t>(params.log_n) ||
      get<uint32_t>(b, 20) != static_cast<uint32_t>(params.prime_count) ||
      get<uint32_t>(b, 24) != static_cast<uint32_t>(params.chain_count) ||
      get<uint32_t>(b, 28) != static_cast<uint32_t>(params.special_prime_count) ||
      get<uint64_t>(b, 32) != chain_hash(params))
    throw std::invalid_argument(fn + ": the object was made by an engine with other parameters.");
  const int type = get<int32_t>(b, 40), flag = get<int32_t>(b, 44);
  const int moduli_id = get<int32_t>(b, 48), polys = get<int32_t>(b, 52);
  const int chains = get<int32_t>(b, 56), delta = get<int32_t>(b, 60);
  if (moduli_id < 0 || moduli_id >= params.chain_count || polys <= 0 ||
      chains != params.chains(moduli_id, (flag & kFlagSpecial) != 0))
    throw std::invalid_argument(fn + ": the object's shape is not valid for this engine.");
  const long double scale =
      static_cast<long double>(get<double>(b, 64)) + static_cast<long double>(get<double>(b, 72));
  const size_t words = static_cast<size_t>(polys) * chains * params.n;
  if (size != kHeaderBytes + words * sizeof(int64_t))
    throw std::invalid_argument(fn + ": the buffer size does not match the object.");
  auto d = upload(type, flag, moduli_id, polys, scale,
                  reinterpret_cast<const int64_t *>(b + kHeaderBytes));
  d->delta = delta;
  synchronize();  // the caller's buffer may be released on return
  return d;
}

}  // namespace fhe_b200
