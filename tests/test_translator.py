"""Unit tests of the Fortran-subset translator (oracle/fortran_subset.py)."""
import os
import subprocess

import pytest

import fortran_subset as fs


PARAMS = """        IMPLICIT REAL*8(A-H,O-Z)
        LOGICAL LFLAG
        PARAMETER(LFLAG=.TRUE.)
        PARAMETER(NA=4,NB=NA+2)
        PARAMETER(SFF=0.4E00)
"""

UNITS = """C a comment line
      SUBROUTINE TEST
        INCLUDE 'p.f'
        DIMENSION A(NB,3)
        COMMON/OUT/A,R1,R2,R3,R4,R5,R6,I1,I2
        DATA ICNT/0/
        R1=1.0E00/3.0E00
        R2=1.0D00/3.0D00
        R3=2.0E00*R1+
     2     1.0E00
        I1=7/2
        I2=-7/2
        R4=(1.0E00/R2)**2
        R5=SFF
        DO 10 K=1,3
        DO 10 J=1,NB
		A(J,K)=FLOAT(J)+10.0E00*FLOAT(K)
10	CONTINUE
        R6=0.0E00
        DO K=1,3
           IF (K.EQ.2) THEN
              R6=R6+A(NB,K)
           ELSE IF (K.EQ.3) THEN
              R6=R6-1.0E00
           ELSE
              R6=R6+0.5E00
           ENDIF
        END DO
        IF (LFLAG) ICNT=ICNT+1
        RETURN
        END
"""


def test_expression_typing():
    sc = fs.Scope(fs.Translator.__new__(fs.Translator), "X")
    tr = sc.tr
    tr.param_types, tr.global_types = {}, {}
    c, t = tr.gen(fs.parse_expr("1.0E00/3.0E00"), sc)
    assert t == "f" and "f" in c
    c, t = tr.gen(fs.parse_expr("1.0D00/3.0E00"), sc)
    assert t == "d"
    c, t = tr.gen(fs.parse_expr("7/2"), sc)
    assert t == "i"
    c, t = tr.gen(fs.parse_expr("X**2"), sc)
    assert c.startswith("ipow_d2")


def test_fixed_form_reading(tmp_path):
    p = tmp_path / "u.f"
    p.write_text(UNITS)
    st = fs.read_fixed_form(str(p))
    texts = [s.text for s in st]
    assert any(t.replace(" ", "").startswith("R3=2.0E00*R1+1.0E00") for t in texts)   # continuation joined
    assert any(s.label == 10 for s in st)


def test_translated_unit_runs(tmp_path):
    (tmp_path / "p.f").write_text(PARAMS)
    (tmp_path / "u.f").write_text(UNITS)
    tr = fs.Translator(str(tmp_path / "p.f"), set())
    code = tr.translate(str(tmp_path / "u.f"), ["TEST"])
    main = r'''
#include "ref_harness.h"
int MPI_COMM_WORLD, MPI_STATUS_SIZE, MPI_DOUBLE_PRECISION, MPI_FLOAT, MPI_MIN, MPI_MAX, MPI_SUM;
int ref_param_override(const char* n, void* d, char t) { (void)n; (void)d; (void)t; return 0; }
void ref_send(void* b, int c, int t, int d, int g) {} void ref_recv(void* b, int c, int t, int d, int g) {}
void ref_sendrecv(void* a, int b, int c, int d, int e, void* f, int g, int h, int i, int j) {}
void ref_allreduce(void* a, void* b, int c, int d, int e) {} void ref_bcast(void* a, int b, int c, int d) {}
void ref_stop(const char* u, int l) { exit(3); } void ref_finalize(void) {}
void sub_STEP(void) {} void sub_FLUXES(void) {} void sub_BCON(void) {} void sub_COMMUNICATE(void) {}
int main(void) {
    ref_params_init(); ref_commons_alloc(); sub_TEST(); sub_TEST();
    printf("%.17g %.17g %.17g %d %d %.17g %.17g %.17g\n", R1, R2, R3, I1, I2, R4, R5, R6);
    printf("%.17g\n", A[(6 - 1) + 6 * (3 - 1)]);
    return 0;
}
'''
    src = tmp_path / "t.c"
    src.write_text(code + main)
    exe = tmp_path / "t"
    here = os.path.dirname(fs.__file__)
    subprocess.run(["gcc", "-O2", "-std=gnu11", "-ffp-contract=off", "-w", "-I", here, "-o", str(exe), str(src), "-lm"],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    import numpy as np
    f13 = float(np.float32(1.0) / np.float32(3.0))
    assert float(out[0]) == f13                      # REAL(4) division widened
    assert float(out[1]) == 1.0 / 3.0                # REAL*8 division
    assert float(out[2]) == 2.0 * f13 + 1.0          # mixed: widened, then double ops
    assert int(out[3]) == 3 and int(out[4]) == -3    # truncating integer division
    assert float(out[5]) == (1.0 / (1.0 / 3.0)) * (1.0 / (1.0 / 3.0))
    assert float(out[6]) == float(np.float32(0.4))   # PARAMETER from a REAL(4) literal
    assert float(out[7]) == 0.5 + (6 + 20.0) - 1.0   # DO/IF/ELSE IF/ELSE, shared DO label
    assert float(out[8]) == 6 + 30.0


def test_unsupported_statement_raises(tmp_path):
    (tmp_path / "p.f").write_text(PARAMS)
    (tmp_path / "u.f").write_text("      SUBROUTINE TEST\n        READ(5,*) X\n        END\n")
    tr = fs.Translator(str(tmp_path / "p.f"), set())
    with pytest.raises(fs.TranslateError):
        tr.translate(str(tmp_path / "u.f"), ["TEST"])
