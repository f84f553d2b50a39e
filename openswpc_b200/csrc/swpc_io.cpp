// swpc_io.cpp -- the reference's on-disk output formats (include/swpc_io.h).
//
// Host code only: SAC / CSF trace files, SAC members of tar archives and
// native .snp v6 snapshot files, laid out byte for byte as the reference's
// Fortran stream writers produce them on a little-endian machine, plus the
// map projection (Gauss-Kruger) that fills the longitude and latitude of
// the headers.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "../../include/swpc_gpu.h"
#include "../../include/swpc_io.h"

namespace {

const double kPi = 3.141592653589793238462643383279502884;   // m_std.f90:14

void blank(char *f, size_t n, const char *s) {
    memset(f, ' ', n);
    if (s) memcpy(f, s, strnlen(s, n));
}

// a Fortran stream write of n bytes; false on a short write
bool put(FILE *fp, const void *p, size_t n) { return fwrite(p, 1, n, fp) == n; }

// octal field of a tar header, Fortran '(O<w>.<w>)': w digits, zero filled
void octal(char *dst, int w, long long v) {
    for (int q = w - 1; q >= 0; q--) {
        dst[q] = (char)('0' + (v & 7));
        v >>= 3;
    }
}

}  // namespace

struct swpc_tar {
    FILE *fp;
};

extern "C" {

void swpc_sac_init(swpc_sac_hdr *h) {
    // sac__init (m_sac.f90:452-562)
    const double ferr = -12345.0;
    const int ierr = -12345;
    double *dd[] = {&h->delta, &h->depmin, &h->depmax, &h->scale, &h->odelta, &h->b, &h->e, &h->o, &h->a, &h->f,
                    &h->stla, &h->stlo, &h->stel, &h->stdp, &h->evla, &h->evlo, &h->evel, &h->evdp, &h->mag,
                    &h->dist, &h->az, &h->baz, &h->gcarc, &h->depmen, &h->cmpaz, &h->cmpinc, &h->xminimum,
                    &h->xmaximum, &h->yminimum, &h->ymaximum};
    for (double *p : dd) *p = ferr;
    for (int q = 0; q < 10; q++) h->t[q] = h->resp[q] = h->user[q] = ferr;
    for (int q = 0; q < 7; q++) h->user_x[q] = ferr;
    int *ii[] = {&h->nzyear, &h->nzjday, &h->nzhour, &h->nzmin, &h->nzsec, &h->nzmsec, &h->norid, &h->nevid,
                 &h->npts, &h->nwfid, &h->nxsize, &h->nysize, &h->idep, &h->iztype, &h->iinst, &h->istreg,
                 &h->ievreg, &h->ievtyp, &h->iqual, &h->isynth, &h->imagtyp, &h->imagsrc};
    for (int *p : ii) *p = ierr;
    for (int q = 0; q < 8; q++) h->iuser[q] = ierr;
    h->nvhdr = 6;
    h->iftype = 1;
    h->leven = 1; h->lpspol = 0; h->lovrok = 1; h->lcalda = 0; h->luser0 = 0;
    const char *c = "-12345";
    blank(h->kstnm, 8, c); blank(h->kevnm, 16, c); blank(h->khole, 8, c); blank(h->ko, 8, c); blank(h->ka, 8, c);
    for (int q = 0; q < 10; q++) blank(h->kt[q], 8, c);
    blank(h->kf, 8, c);
    for (int q = 0; q < 3; q++) blank(h->kuser[q], 8, c);
    blank(h->kcmpnm, 8, c); blank(h->knetwk, 8, c); blank(h->kdatrd, 8, c); blank(h->kinst, 8, c);
    h->nzmonth = h->nzday = h->tim = 0;
}

void swpc_sac_header_bytes(const swpc_sac_hdr *h, unsigned char out[632]) {
    // sac__whdr (m_sac.f90:314-449): words not copied keep their undefined values
    float fh[70];
    int ih[35], lh[5];
    char ah[48][4];
    for (float &v : fh) v = -12345.0f;
    for (int &v : ih) v = -12345;
    for (int &v : lh) v = 0;
    for (int q = 0; q < 48; q += 2) {
        memcpy(ah[q], "-123", 4);
        memcpy(ah[q + 1], "45  ", 4);
    }
    auto F = [&](int word, double v) { fh[word - 1] = (float)v; };
    fh[0] = (float)(int)(h->delta * 1e7) / 1e7f;   // delta truncated to 1e-7 (word 1)
    F(2, h->depmin); F(3, h->depmax); F(6, h->b); F(7, h->e); F(8, h->o); F(9, h->a);
    for (int q = 0; q < 10; q++) F(11 + q, h->t[q]);
    F(32, h->stla); F(33, h->stlo); F(34, h->stel); F(35, h->stdp); F(36, h->evla); F(37, h->evlo);
    F(38, h->evel); F(39, h->evdp); F(40, h->mag);
    for (int q = 0; q < 10; q++) F(41 + q, h->user[q]);
    F(51, h->dist); F(52, h->az); F(53, h->baz); F(54, h->gcarc); F(57, h->depmen); F(58, h->cmpaz);
    F(59, h->cmpinc);
    for (int q = 0; q < 7; q++) F(64 + q, h->user_x[q]);
    auto I = [&](int word, int v) { ih[word - 71] = v; };
    I(71, h->nzyear); I(72, h->nzjday); I(73, h->nzhour); I(74, h->nzmin); I(75, h->nzsec); I(76, h->nzmsec);
    I(77, h->nvhdr); I(80, h->npts); I(86, h->iftype); I(87, h->idep); I(93, h->ievtyp);
    for (int q = 0; q < 8; q++) I(98 + q, h->iuser[q]);
    lh[0] = h->leven ? 1 : 0; lh[1] = h->lpspol ? 1 : 0; lh[2] = h->lovrok ? 1 : 0; lh[3] = h->lcalda ? 1 : 0;
    lh[4] = h->luser0 ? 1 : 0;
    // words 111-158: two 4-byte words per 8-character field, kevnm four
    const char *k8[] = {h->khole, h->ko, h->ka, h->kt[0], h->kt[1], h->kt[2], h->kt[3], h->kt[4], h->kt[5],
                        h->kt[6], h->kt[7], h->kt[8], h->kt[9], h->kf, h->kuser[0], h->kuser[1], h->kuser[2],
                        h->kcmpnm, h->knetwk, h->kdatrd, h->kinst};
    memcpy(ah[0], h->kstnm, 8);
    memcpy(ah[2], h->kevnm, 16);
    for (int q = 0; q < 21; q++) memcpy(ah[6 + 2 * q], k8[q], 8);
    memcpy(out, fh, 280);
    memcpy(out + 280, ih, 140);
    memcpy(out + 420, lh, 20);
    memcpy(out + 440, ah, 192);
}

int swpc_sac_write(const char *path, const swpc_sac_hdr *h, const float *data) {
    if (!path || !h || (h->npts > 0 && !data) || h->npts < 0) return SWPC_ERR_ARG;
    FILE *fp = fopen(path, "wb");
    if (!fp) return SWPC_ERR_IO;
    unsigned char hb[632];
    swpc_sac_header_bytes(h, hb);
    bool ok = put(fp, hb, sizeof(hb)) && put(fp, data, sizeof(float) * (size_t)h->npts);
    ok = (fclose(fp) == 0) && ok;
    return ok ? SWPC_OK : SWPC_ERR_IO;
}

int swpc_csf_write(const char *path, int ntrace, int npts, const swpc_sac_hdr *h, const float *data) {
    if (!path || ntrace < 0 || npts < 0 || (ntrace > 0 && (!h || !data))) return SWPC_ERR_ARG;
    for (int n = 0; n < ntrace; n++)
        if (h[n].npts != npts) return SWPC_ERR_ARG;   // wcsf_s refuses a npts mismatch
    FILE *fp = fopen(path, "wb");
    if (!fp) return SWPC_ERR_IO;
    bool ok = put(fp, "CSFD", 4) && put(fp, &ntrace, 4) && put(fp, &npts, 4);
    unsigned char hb[632];
    for (int n = 0; n < ntrace && ok; n++) {
        swpc_sac_header_bytes(&h[n], hb);
        ok = put(fp, hb, sizeof(hb)) && put(fp, data + (size_t)n * npts, sizeof(float) * (size_t)npts);
    }
    ok = (fclose(fp) == 0) && ok;
    return ok ? SWPC_OK : SWPC_ERR_IO;
}

swpc_tar *swpc_tar_open(const char *path) {
    if (!path) return nullptr;
    FILE *fp = fopen(path, "wb");
    if (!fp) return nullptr;
    swpc_tar *t = new swpc_tar;
    t->fp = fp;
    return t;
}

int swpc_tar_add_sac(swpc_tar *t, const char *name, const swpc_sac_hdr *h, const float *data) {
    if (!t || !name || !h || h->npts < 0 || (h->npts > 0 && !data)) return SWPC_ERR_ARG;
    const size_t ln = strlen(name);
    if (ln > 99) return SWPC_ERR_ARG;
    // tar__whdr (m_tar.f90): the block starts as one NUL followed by blanks (a Fortran character assignment);
    // every text field is written with a trailing NUL, numbers as zero-filled octal without terminator
    char b[512];
    memset(b, ' ', sizeof(b));
    b[0] = '\0';
    memcpy(b, name, ln);
    b[ln] = '\0';
    const long long fsize = (158LL + h->npts) * 4;
    octal(b + 100, 8, 420);     // mode 0644
    octal(b + 108, 8, 0);       // uid
    octal(b + 116, 8, 0);       // gid
    octal(b + 124, 12, fsize);
    octal(b + 136, 12, h->tim); // mtime
    b[156] = '0';               // typeflag
    b[157] = '\0'; b[158] = '\0';                  // linkname (empty)
    memcpy(b + 257, "ustar", 5); b[262] = '\0';   // magic
    memcpy(b + 265, "root", 4); b[269] = '\0';    // uname
    memcpy(b + 297, "root", 4); b[301] = '\0';    // gname
    b[329] = b[330] = '\0';                        // devmajor
    b[337] = b[338] = '\0';                        // devminor
    b[345] = b[346] = '\0';                        // prefix
    long long sum = 0;                             // with the checksum field blank
    for (unsigned char c : b) sum += c;
    octal(b + 148, 8, sum);
    unsigned char hb[632];
    swpc_sac_header_bytes(h, hb);
    static const char zeros[512] = {0};
    const int m = (int)(fsize % 512);              // tar__wpad: 512 - m NULs, a whole block when m = 0
    bool ok = put(t->fp, b, 512) && put(t->fp, hb, sizeof(hb)) &&
              put(t->fp, data, sizeof(float) * (size_t)h->npts) && put(t->fp, zeros, 512 - m);
    return ok ? SWPC_OK : SWPC_ERR_IO;
}

int swpc_tar_close(swpc_tar *t) {
    if (!t) return SWPC_ERR_ARG;
    static const char zeros[1024] = {0};
    bool ok = put(t->fp, zeros, sizeof(zeros));   // tar__wend
    ok = (fclose(t->fp) == 0) && ok;
    delete t;
    return ok ? SWPC_OK : SWPC_ERR_IO;
}

int swpc_snp_write(const char *path, const swpc_snp_hdr *h, int nmed_written, const float *med, int nframes,
                   const float *frames) {
    if (!path || !h || h->ns1 < 1 || h->ns2 < 1 || nmed_written < 0 || nframes < 0 || h->nsnp < 1 ||
        (nmed_written > 0 && !med) || (nframes > 0 && !frames))
        return SWPC_ERR_ARG;
    FILE *fp = fopen(path, "wb");
    if (!fp) return SWPC_ERR_IO;
    const int version = 6;
    const float dum = 1.0f;
    // write_snp_header (m_snap.f90:838-884)
    bool ok = put(fp, "STREAMIO", 8) && put(fp, "SWPC_3D ", 8) && put(fp, &version, 4) && put(fp, h->title, 80) &&
              put(fp, &h->exedate, 4) && put(fp, h->coordinate, 2) && put(fp, h->snaptype, 2) &&
              put(fp, &h->ns1, 4) && put(fp, &h->ns2, 4) && put(fp, &h->xs1, 4) && put(fp, &h->xs2, 4) &&
              put(fp, &h->ds1, 4) && put(fp, &h->ds2, 4) && put(fp, &h->dt, 4) && put(fp, &h->na1, 4) &&
              put(fp, &h->na2, 4) && put(fp, &h->nmed, 4) && put(fp, &h->nsnp, 4) && put(fp, &h->clon, 4) &&
              put(fp, &h->clat, 4) && put(fp, &h->phi, 4) && put(fp, &dum, 4) && put(fp, &dum, 4) &&
              put(fp, &dum, 4);
    const size_t plane = (size_t)h->ns1 * h->ns2;
    if (ok) ok = put(fp, med, sizeof(float) * plane * nmed_written);
    if (ok) ok = put(fp, frames, sizeof(float) * plane * h->nsnp * nframes);
    ok = (fclose(fp) == 0) && ok;
    return ok ? SWPC_OK : SWPC_ERR_IO;
}

void swpc_geomap_c2g(float x, float y, float clon, float clat, float phi, float *lon, float *lat) {
    // rotation by phi in single precision (m_geomap.f90:59-61)
    const float phr = (float)(kPi / 180.0 * (double)phi);
    const float xx = cosf(phr) * x - sinf(phr) * y;
    const float yy = sinf(phr) * x + cosf(phr) * y;
    // Gauss-Kruger inverse (xytoll_d, m_gk.f90): GRS80 (a = 6378137 m, 1/f = 298.257222101), scale 0.9999,
    // Kruger series in the third flattening n
    const double a = 6378137.0, F = 298.257222101, m0 = 0.9999, n = 1.0 / (2.0 * F - 1.0);
    double beta[5], delta[6], AA[6];
    beta[0] = (1 / 2. + (-2 / 3. + (37 / 96. + (-1 / 360. - 81 / 512. * n) * n) * n) * n) * n;
    beta[1] = ((1 / 48. + (1 / 15. + (-437 / 1440. + 46 / 105. * n) * n) * n) * n) * n;
    beta[2] = (((17 / 480. + (-37 / 840. - 209 / 4480. * n) * n) * n) * n) * n;
    beta[3] = ((((4397 / 161280. - 11 / 504. * n) * n) * n) * n) * n;
    beta[4] = ((((4583 / 161280. * n) * n) * n) * n) * n;
    delta[0] = (2 / 1. + (-2 / 3. + (-2 / 1. + (116 / 45. + (26 / 45. + (-2854 / 675.) * n) * n) * n) * n) * n) * n;
    delta[1] = ((7 / 3. + (-8 / 5. + (-227 / 45. + (2704 / 315. + (2323 / 945.) * n) * n) * n) * n) * n) * n;
    delta[2] = (((56 / 15. + (-136 / 35. + (-1262 / 105. + (73814 / 2835.) * n) * n) * n) * n) * n) * n;
    delta[3] = ((((4279 / 630. + (-332 / 35. + (-399572 / 14175.) * n) * n) * n) * n) * n) * n;
    delta[4] = (((((4174 / 315. + (-144838 / 6237.) * n) * n) * n) * n) * n) * n;
    delta[5] = ((((((601676 / 22275.) * n) * n) * n) * n) * n) * n;
    const double n2 = n * n, n3 = n2 * n, n4 = n2 * n2, n5 = n4 * n;   // integer powers n**k
    AA[0] = 1 + (1 / 4. + 1 / 64. * n2) * n2;
    AA[1] = -3 / 2. * (1. - 1 / 8. * n2 - 1 / 64. * n4) * n;
    AA[2] = 15 / 16. * (1. - 1 / 4. * n2) * n2;
    AA[3] = -35 / 48. * (1. - 5 / 16. * n2) * n3;
    AA[4] = 315 / 512. * n4;
    AA[5] = -693 / 1280. * n5;
    const double lam0 = kPi / 180.0 * (double)clon, phi0 = kPi / 180.0 * (double)clat;
    const double Abar = m0 * a / (1 + n) * AA[0];
    double s = AA[0] * phi0;
    for (int j = 1; j <= 5; j++) s = s + AA[j] * sin(2 * j * phi0);
    s = s * (m0 * a / (1 + n));
    const double xi = ((double)xx * 1000 + s) / Abar, eta = (double)yy * 1000 / Abar;
    double xi2 = xi, eta2 = eta;
    for (int j = 1; j <= 5; j++) {
        xi2 = xi2 - beta[j - 1] * sin(2 * j * xi) * cosh(2 * j * eta);
        eta2 = eta2 - beta[j - 1] * cos(2 * j * xi) * sinh(2 * j * eta);
    }
    const double chi = asin(sin(xi2) / cosh(eta2));
    const double lam = lam0 + atan(sinh(eta2) / cos(xi2));
    double ph = chi;
    for (int j = 1; j <= 6; j++) ph = ph + delta[j - 1] * sin(2 * j * chi);
    *lon = (float)(180.0 / kPi * lam);
    *lat = (float)(180.0 / kPi * ph);
}

}  // extern "C"
