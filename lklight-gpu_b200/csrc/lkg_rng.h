// rand 0.7.3 StdRng stream (the GSO's and the setup's random numbers).
//
// StdRng is ChaCha20 (rand_chacha 0.2: 20 rounds, 64-bit block counter,
// stream id 0, four blocks buffered), seeded by rand_core 0.5.1
// seed_from_u64, which fills the 256-bit key with eight PCG32 (XSH-RR)
// outputs.  gen::<f64>() takes the top 53 bits of next_u64 (low word first)
// times 2^-53.  Written from the published ChaCha20 and PCG32 definitions;
// pinned by the reference's seeded-quaternion test (qt.rs:474-488).
#pragma once
#include <cstdint>
#include <cstring>

namespace lkg {

class StdRng {
  public:
    explicit StdRng(uint64_t seed = 0) { seed_from_u64(seed); }

    void seed_from_u64(uint64_t state) {
        for (int i = 0; i < 8; ++i) {
            state = state * 6364136223846793005ull + 11634580027462260723ull;
            uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
            uint32_t rot = (uint32_t)(state >> 59);
            key_[i] = (xs >> rot) | (xs << ((32u - rot) & 31u));
        }
        ctr_ = 0;
        idx_ = 64;
    }

    uint64_t next_u64() {
        if (idx_ >= 64) refill();
        if (idx_ == 63) {
            uint64_t lo = buf_[63];
            refill();
            idx_ = 1;
            return ((uint64_t)buf_[0] << 32) | lo;
        }
        uint64_t v = ((uint64_t)buf_[idx_ + 1] << 32) | buf_[idx_];
        idx_ += 2;
        return v;
    }

    double gen_f64() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }

    // position in the keystream, in 32-bit words consumed since seeding
    // (the device GSO draws word pairs 2i, 2i + 1 for draw i directly)
    uint64_t words_used() const { return idx_ >= 64 ? ctr_ * 16 : (ctr_ - 4) * 16 + (uint64_t)idx_; }
    void set_words_used(uint64_t w) {
        if (w % 64 == 0) {
            ctr_ = w / 16;
            idx_ = 64;
        } else {
            ctr_ = (w / 64) * 4;
            refill();
            idx_ = (int)(w % 64);
        }
    }
    const uint32_t* key() const { return key_; }

  private:
    static uint32_t rotl(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }

    void block(uint64_t ctr, uint32_t* out) const {
        uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key_[0], key_[1], key_[2], key_[3],
                          key_[4], key_[5], key_[6], key_[7], (uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 0u};
        uint32_t x[16];
        memcpy(x, s, sizeof(x));
        auto qr = [&](int a, int b, int c, int d) {
            x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 16);
            x[c] += x[d]; x[b] = rotl(x[b] ^ x[c], 12);
            x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 8);
            x[c] += x[d]; x[b] = rotl(x[b] ^ x[c], 7);
        };
        for (int r = 0; r < 10; ++r) {
            qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
            qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
        }
        for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
    }

    void refill() {
        for (int b = 0; b < 4; ++b) block(ctr_ + b, buf_ + 16 * b);
        ctr_ += 4;
        idx_ = 0;
    }

    uint32_t key_[8];
    uint64_t ctr_ = 0;
    uint32_t buf_[64];
    int idx_ = 64;
};

}  // namespace lkg
