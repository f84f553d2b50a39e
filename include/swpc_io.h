/*
 * swpc_io.h -- on-disk output formats of the B200 OpenSWPC library.
 *
 * The time step hands traces (swpc_wav_fetch) and snapshot frames
 * (swpc_snap_fetch) over in memory; these routines write them in the
 * reference's file formats, byte for byte as its writers lay them out:
 *   SAC       one trace per file (sac__write / sac__whdr,
 *             src/shared/m_sac.f90:267-449), machine endian, header version 6;
 *   CSF       all traces of a run in one file ('CSFD', ntrace, npts, then
 *             header + data per trace; csf__write, m_sac.f90:585-648);
 *   tar       SAC files bundled in a tar archive (sac__wtar with the ustar
 *             header of m_tar.f90's tar__whdr / tar__wpad / tar__wend);
 *   .snp v6   native snapshot files: the fixed header of write_snp_header
 *             (src/swpc_3d/m_snap.f90:838-884), the medium planes of
 *             newfile_yz / newfile_xz / newfile_xy (:324-473), then every
 *             frame's arrays in order.
 * A Fortran driver that keeps the reference's own writers needs none of
 * this; these serve C, C++ and Python drivers.  Every call returns 0 or
 * SWPC_ERR_ARG (bad arguments) / SWPC_ERR_IO (the file could not be written).
 */
#ifndef SWPC_IO_H
#define SWPC_IO_H

#ifdef __cplusplus
extern "C" {
#endif

#define SWPC_ERR_IO 7

/* sac__hdr (m_sac.f90:21-156).  Character fields are blank padded, not NUL
 * terminated, as Fortran stores them. */
typedef struct swpc_sac_hdr {
    double delta, depmin, depmax, scale, odelta, b, e, o, a;
    double t[10];
    double f;
    double resp[10];
    double stla, stlo, stel, stdp, evla, evlo, evel, evdp, mag;
    double user[10];
    double dist, az, baz, gcarc, depmen, cmpaz, cmpinc;
    double xminimum, xmaximum, yminimum, ymaximum;
    double user_x[7];                /* user10..user16 (header words 64-70) */
    int nzyear, nzjday, nzhour, nzmin, nzsec, nzmsec, nvhdr, norid, nevid, npts, nwfid, nxsize, nysize;
    int iftype, idep, iztype, iinst, istreg, ievreg, ievtyp, iqual, isynth, imagtyp, imagsrc;
    int iuser[8];                    /* words 98-105 */
    int leven, lpspol, lovrok, lcalda, luser0;
    char kstnm[8], kevnm[16], khole[8], ko[8], ka[8], kt[10][8], kf[8], kuser[3][8];
    char kcmpnm[8], knetwk[8], kdatrd[8], kinst[8];
    int nzmonth, nzday, tim;         /* date of the run and its POSIX time (tar mtime) */
} swpc_sac_hdr;

/* sac__init (m_sac.f90:452-562): every field undefined (-12345), nvhdr 6,
 * iftype 1, leven and lovrok true. */
void swpc_sac_init(swpc_sac_hdr *h);
/* The 632-byte binary header sac__whdr writes (words 1-158). */
void swpc_sac_header_bytes(const swpc_sac_hdr *h, unsigned char out[632]);
/* One SAC file: header + h->npts samples (replaces an existing file). */
int swpc_sac_write(const char *path, const swpc_sac_hdr *h, const float *data);
/* One CSF file of ntrace traces of npts samples: data(npts, ntrace). */
int swpc_csf_write(const char *path, int ntrace, int npts, const swpc_sac_hdr *h, const float *data);

/* tar archives of SAC files (wav_format 'tar_st' / 'tar_node'). */
typedef struct swpc_tar swpc_tar;
swpc_tar *swpc_tar_open(const char *path);
/* One member: a ustar header for `name` with mtime h->tim, the SAC header and
 * data, NUL padding as tar__wpad writes it. */
int swpc_tar_add_sac(swpc_tar *t, const char *name, const swpc_sac_hdr *h, const float *data);
/* tar__wend's two zero blocks, then the file is closed. */
int swpc_tar_close(swpc_tar *t);

/* The fixed header of a native snapshot file (write_snp_header). */
typedef struct swpc_snp_hdr {
    char title[80];                  /* blank padded */
    int exedate;                     /* POSIX time of the run */
    char coordinate[2];              /* yz xz xy fs ob */
    char snaptype[2];                /* ps v3 u3 */
    int ns1, ns2;                    /* plane size */
    float xs1, xs2;                  /* first sample coordinates */
    float ds1, ds2;                  /* sample spacing along each axis */
    float dt;                        /* dt * ntdec_s */
    int na1, na2;                    /* absorber width in samples */
    int nmed, nsnp;                  /* medium and snapshot arrays per plane */
    float clon, clat, phi;           /* map projection of the grid */
} swpc_snp_hdr;
/* A complete native snapshot file: header, nmed_written medium planes
 * med(ns1, ns2, nmed_written) and nframes frames frames(ns1, ns2, nsnp,
 * nframes), all Fortran order. */
int swpc_snp_write(const char *path, const swpc_snp_hdr *h, int nmed_written, const float *med, int nframes,
                   const float *frames);

/* geomap__c2g (src/shared/m_geomap.f90:44-65): grid coordinates x (north),
 * y (east) [km] about the centre (clon, clat) rotated by phi [deg] to
 * longitude and latitude, through the Gauss-Kruger inverse projection of
 * src/shared/m_gk.f90 (Kruger series to the 6th order, GRS80). */
void swpc_geomap_c2g(float x, float y, float clon, float clat, float phi, float *lon, float *lat);

#ifdef __cplusplus
}
#endif
#endif
