// Fortran 'binary' dumps of the state (output.f90:224-235, read back by restart.f90:212-221).
//
// The file is four header records and the uin record, written as gfortran writes an
// unformatted sequential file: every record is framed by 4-byte length markers.  A
// record longer than kMaxSubrecord bytes is split into subrecords, each framed by its
// own markers; a negative leading marker says that another subrecord follows and a
// negative trailing marker that one precedes (the gfortran manual's description of its
// unformatted sequential format).  Records:
//   1  int32  nx, ny, nz, nxslice, nyslice, nzslice
//   2  double time, dt, dx, dy, dz
//   3  double xmin, xmax, ymin, ymax, zmin, zmax
//   4  double gamma, ciso
//   5  double uin(iu1:iu2, ju1:ju2, ku1:ku2, 1:11), Fortran order
// Host code only; the device side streams the uin record plane by plane through it.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

namespace dg {
namespace dump {

constexpr long long kMaxSubrecord = 2147483639LL;  // 2 GiB - 9, with 4-byte markers

struct Header {
    int32_t nx, ny, nz, nxslice, nyslice, nzslice;
    double time, dt, dx, dy, dz;
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double gamma, ciso;
};

// writes one logical record of a known total length, in as many write() calls as wanted
class RecordWriter {
  public:
    RecordWriter(FILE *f, long long total, long long max_sub = kMaxSubrecord)
        : f_(f), remaining_(total), max_sub_(max_sub) { start(); }
    bool write(const void *data, long long n) {
        const char *p = static_cast<const char *>(data);
        while (n > 0 && ok_) {
            if (remaining_ <= 0) { ok_ = false; break; }  // more bytes than announced
            if (sub_done_ == sub_len_) finish_sub();
            const long long k = n < sub_len_ - sub_done_ ? n : sub_len_ - sub_done_;
            if ((long long)std::fwrite(p, 1, (size_t)k, f_) != k) ok_ = false;
            p += k;
            n -= k;
            sub_done_ += k;
            remaining_ -= k;
        }
        return ok_;
    }
    // closes the last subrecord; false if fewer or more bytes than announced were written
    bool close() {
        if (!ok_ || remaining_ != 0 || sub_done_ != sub_len_) return false;
        marker(sub_index_ > 0 ? -sub_len_ : sub_len_);
        return ok_;
    }

  private:
    void start() {
        sub_len_ = remaining_ < max_sub_ ? remaining_ : max_sub_;
        sub_done_ = 0;
        marker(remaining_ > sub_len_ ? -sub_len_ : sub_len_);
    }
    void finish_sub() {  // a full subrecord with data still to come
        marker(sub_index_ > 0 ? -sub_len_ : sub_len_);
        sub_index_++;
        start();
    }
    void marker(long long v) {
        const int32_t m = (int32_t)v;
        if (std::fwrite(&m, 4, 1, f_) != 1) ok_ = false;
    }
    FILE *f_;
    long long remaining_, max_sub_, sub_len_ = 0, sub_done_ = 0;
    int sub_index_ = 0;
    bool ok_ = true;
};

// reads one logical record whose total length the caller knows
class RecordReader {
  public:
    explicit RecordReader(FILE *f) : f_(f) { next(); }
    bool read(void *data, long long n) {
        char *p = static_cast<char *>(data);
        while (n > 0 && ok_) {
            if (sub_done_ == sub_len_) {
                if (!more_) { ok_ = false; break; }  // the record is shorter than expected
                if (!trailer()) break;
                next();
                continue;
            }
            const long long k = n < sub_len_ - sub_done_ ? n : sub_len_ - sub_done_;
            if ((long long)std::fread(p, 1, (size_t)k, f_) != k) ok_ = false;
            p += k;
            n -= k;
            sub_done_ += k;
        }
        return ok_;
    }
    // the whole record has been consumed: no bytes left and no further subrecord
    bool close() {
        if (!ok_ || sub_done_ != sub_len_ || more_) return false;
        return trailer();
    }

  private:
    void next() {
        int32_t m;
        if (std::fread(&m, 4, 1, f_) != 1) { ok_ = false; return; }
        more_ = m < 0;
        sub_len_ = m < 0 ? -(long long)m : (long long)m;
        sub_done_ = 0;
    }
    bool trailer() {
        int32_t m;
        if (std::fread(&m, 4, 1, f_) != 1) return ok_ = false;
        const long long len = m < 0 ? -(long long)m : (long long)m;
        if (len != sub_len_ || (m < 0) != (index_ > 0)) return ok_ = false;
        index_++;
        return true;
    }
    FILE *f_;
    long long sub_len_ = 0, sub_done_ = 0;
    int index_ = 0;
    bool more_ = false, ok_ = true;
};

inline bool write_header(FILE *f, const Header &h) {
    const int32_t ints[6] = {h.nx, h.ny, h.nz, h.nxslice, h.nyslice, h.nzslice};
    const double r2[5] = {h.time, h.dt, h.dx, h.dy, h.dz};
    const double r3[6] = {h.xmin, h.xmax, h.ymin, h.ymax, h.zmin, h.zmax};
    const double r4[2] = {h.gamma, h.ciso};
    RecordWriter a(f, sizeof ints);
    if (!a.write(ints, sizeof ints) || !a.close()) return false;
    RecordWriter b(f, sizeof r2);
    if (!b.write(r2, sizeof r2) || !b.close()) return false;
    RecordWriter c(f, sizeof r3);
    if (!c.write(r3, sizeof r3) || !c.close()) return false;
    RecordWriter d(f, sizeof r4);
    return d.write(r4, sizeof r4) && d.close();
}

inline bool read_header(FILE *f, Header &h) {
    int32_t ints[6];
    double r2[5], r3[6], r4[2];
    RecordReader a(f);
    if (!a.read(ints, sizeof ints) || !a.close()) return false;
    RecordReader b(f);
    if (!b.read(r2, sizeof r2) || !b.close()) return false;
    RecordReader c(f);
    if (!c.read(r3, sizeof r3) || !c.close()) return false;
    RecordReader d(f);
    if (!d.read(r4, sizeof r4) || !d.close()) return false;
    h.nx = ints[0]; h.ny = ints[1]; h.nz = ints[2];
    h.nxslice = ints[3]; h.nyslice = ints[4]; h.nzslice = ints[5];
    h.time = r2[0]; h.dt = r2[1]; h.dx = r2[2]; h.dy = r2[3]; h.dz = r2[4];
    h.xmin = r3[0]; h.xmax = r3[1]; h.ymin = r3[2]; h.ymax = r3[3]; h.zmin = r3[4]; h.zmax = r3[5];
    h.gamma = r4[0]; h.ciso = r4[1];
    return true;
}

}  // namespace dump
}  // namespace dg
