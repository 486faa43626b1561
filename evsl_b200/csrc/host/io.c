/*
 * io.c -- matrix ingestion: Matrix-Market coordinate files and COO -> CSR
 * on the device.
 *
 * evslx_read_coo_MM follows the reference drivers' reader read_coo_MM
 * (TESTS/COMMON/io.c:115-214, with the banner and size rules of
 * TESTS/COMMON/mmio.c:80-210): real or integer coordinate matrices, square,
 * symmetric files expanded by appending the transposed off-diagonal entries
 * after the stored ones (in file order), indices shifted by idxout - idxin.
 * Differences: a file that cannot be opened returns EVSLX_ERR_ARG instead of
 * exiting; entries may be separated by any white space; indices are parsed
 * exactly (the reference passes them through a float, which is exact below
 * 2^24 only).
 */
#include <ctype.h>
#include <errno.h>

#include "internal.h"

static void lower(char *s) {
  for (; *s; s++) *s = (char)tolower((unsigned char)*s);
}

int evslx_read_coo_MM(const char *matfile, int idxin, int idxout, cooMat *Acoo) {
  if (!matfile || !Acoo) return evsl_seterr(EVSLX_ERR_ARG, "evslx_read_coo_MM: null argument");
  FILE *f = fopen(matfile, "r");
  if (!f) return evsl_seterr(EVSLX_ERR_ARG, "unable to open matrix file %s", matfile);
  char line[1100], banner[64], obj[64], fmt[64], field[64], sym[64];
  int rc = 1;
  int nrow = 0, ncol = 0, nnz = 0;
  int *IR = NULL, *JC = NULL;
  double *VAL = NULL;
  char *buf = NULL;
  /* banner: %%MatrixMarket matrix coordinate real|integer general|symmetric|... */
  if (!fgets(line, sizeof(line), f) ||
      sscanf(line, "%63s %63s %63s %63s %63s", banner, obj, fmt, field, sym) != 5 ||
      strncmp(banner, "%%MatrixMarket", 14) != 0) {
    evsl_seterr(1, "%s: could not process the Matrix Market banner", matfile);
    goto out;
  }
  lower(obj);
  lower(fmt);
  lower(field);
  lower(sym);
  const int symmetric = strcmp(sym, "symmetric") == 0;
  if (strcmp(obj, "matrix") != 0 || strcmp(fmt, "coordinate") != 0 ||
      (strcmp(field, "real") != 0 && strcmp(field, "integer") != 0) ||
      (!symmetric && strcmp(sym, "general") != 0 && strcmp(sym, "skew-symmetric") != 0)) {
    evsl_seterr(1, "%s: only sparse real-valued/integer coordinate matrices are supported", matfile);
    goto out;
  }
  /* size line after the comments */
  do {
    if (!fgets(line, sizeof(line), f)) {
      evsl_seterr(1, "%s: missing size line", matfile);
      goto out;
    }
  } while (line[0] == '%');
  if (sscanf(line, "%d %d %d", &nrow, &ncol, &nnz) != 3) {
    do {
      const int got = fscanf(f, "%d %d %d", &nrow, &ncol, &nnz);
      if (got == EOF) {
        evsl_seterr(1, "%s: missing size line", matfile);
        goto out;
      }
      if (got == 3) break;
    } while (1);
  }
  if (nrow != ncol) {
    evsl_seterr(1, "%s: not a square matrix (%d x %d)", matfile, nrow, ncol);
    goto out;
  }
  if (nrow < 0 || nnz < 0 || (symmetric && nnz > 0x3fffffff)) {
    evsl_seterr(1, "%s: bad sizes (%d, %d)", matfile, nrow, nnz);
    goto out;
  }
  const size_t cap = symmetric ? 2 * (size_t)nnz : (size_t)nnz;
  IR = (int *)malloc(sizeof(int) * (cap ? cap : 1));
  JC = (int *)malloc(sizeof(int) * (cap ? cap : 1));
  VAL = (double *)malloc(sizeof(double) * (cap ? cap : 1));
  /* the entries: read the rest of the file once and parse it in place */
  const long here = ftell(f);
  fseek(f, 0, SEEK_END);
  const long end = ftell(f);
  fseek(f, here, SEEK_SET);
  const size_t len = (end > here) ? (size_t)(end - here) : 0;
  buf = (char *)malloc(len + 1);
  if (!IR || !JC || !VAL || !buf) {
    rc = evsl_seterr(EVSLX_ERR_NOMEM, "%s: out of host memory", matfile);
    goto out;
  }
  const size_t got = fread(buf, 1, len, f);
  buf[got] = '\0';
  char *p = buf, *q;
  for (int k = 0; k < nnz; k++) {
    const double r = strtod(p, &q);
    if (q == p) goto truncated;
    p = q;
    const double c = strtod(p, &q);
    if (q == p) goto truncated;
    p = q;
    const double v = strtod(p, &q);
    if (q == p) goto truncated;
    p = q;
    IR[k] = (int)r;
    JC[k] = (int)c;
    VAL[k] = v;
  }
  int total = nnz;
  if (symmetric) {
    for (int k = 0; k < nnz; k++) {
      if (IR[k] != JC[k]) {
        IR[total] = JC[k];
        JC[total] = IR[k];
        VAL[total] = VAL[k];
        total++;
      }
    }
  }
  const int offset = idxout - idxin;
  if (offset) {
    for (int i = 0; i < total; i++) {
      IR[i] += offset;
      JC[i] += offset;
    }
  }
  Acoo->nrows = nrow;
  Acoo->ncols = ncol;
  Acoo->nnz = total;
  Acoo->ir = IR;
  Acoo->jc = JC;
  Acoo->vv = VAL;
  IR = JC = NULL;
  VAL = NULL;
  rc = 0;
  goto out;
truncated:
  rc = -1;
  evsl_seterr(-1, "%s: fewer than %d entries", matfile, nnz);
out:
  fclose(f);
  free(buf);
  free(IR);
  free(JC);
  free(VAL);
  return rc;
}

int evslx_coo_to_csr_device(int cooidx, const cooMat *coo, int coo_on_device, csrMat *Agpu) {
  if (!coo || !Agpu || coo->nrows <= 0 || coo->nrows != coo->ncols || coo->nnz < 0)
    return evsl_seterr(EVSLX_ERR_ARG, "evslx_coo_to_csr_device: need a square COO matrix");
  if (!evslh.started) return evsl_seterr(EVSLX_ERR_STATE, "evslx_coo_to_csr_device: call EVSLStart first");
  const int n = coo->nrows, nnz = coo->nnz;
  const int *ir = coo->ir, *jc = coo->jc;
  const double *vv = coo->vv;
  int *dir = NULL, *djc = NULL;
  double *dvv = NULL;
  int rc = 0;
  if (!coo_on_device && nnz > 0) {
    dir = (int *)evslcu_malloc(sizeof(int) * (size_t)nnz);
    djc = (int *)evslcu_malloc(sizeof(int) * (size_t)nnz);
    dvv = (double *)evslcu_malloc(sizeof(double) * (size_t)nnz);
    if (!dir || !djc || !dvv || evslcu_h2d(dir, ir, sizeof(int) * (size_t)nnz) ||
        evslcu_h2d(djc, jc, sizeof(int) * (size_t)nnz) || evslcu_h2d(dvv, vv, sizeof(double) * (size_t)nnz))
      rc = EVSLCU_ERR_NOMEM;
    ir = dir;
    jc = djc;
    vv = dvv;
  }
  int *ia = NULL, *ja = NULL;
  double *a = NULL;
  if (!rc) rc = evslcu_coo_to_csr(n, nnz, ir, jc, vv, cooidx, &ia, &ja, &a);
  evslcu_free(dir);
  evslcu_free(djc);
  evslcu_free(dvv);
  if (rc) return evsl_seterr(rc, "%s", evslcu_errstr());
  Agpu->owndata = 2;
  Agpu->nrows = n;
  Agpu->ncols = n;
  Agpu->nnz = nnz;
  Agpu->ia = ia;
  Agpu->ja = ja;
  Agpu->a = a;
  Agpu->descr = NULL;
  Agpu->dBuffer = NULL;
  return 0;
}
