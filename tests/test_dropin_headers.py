"""Drop-in header check (CPU): the reference's own QFunction sources and a HONEE-style operator set-up compile and link
against include/ceed/*.h and libceed_b200.so, so `navierstokes` can be rebuilt against this backend unchanged."""
import os
import subprocess
import textwrap

import pytest
from helpers import reference_dir

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
INC = os.path.join(ROOT, "include")
REF = reference_dir()


@pytest.mark.skipif(REF is None, reason="reference sources not present (set HONEE_REFERENCE_DIR)")
@pytest.mark.parametrize("header", ["newtonian.h", "setupgeo.h", "taylorgreen.h", "monitor_totalkineticenergy.h"])
def test_reference_qfunctions_compile_against_our_headers(tmp_path, header):
    src = tmp_path / "t.c"
    src.write_text(f'#include <ceed.h>\n#include "{header}"\nint main(void) {{ return 0; }}\n')
    r = subprocess.run(["gcc", "-std=gnu99", "-fsyntax-only", "-Wno-unused-function", f"-I{INC}", f"-I{REF}/qfunctions", str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]


def test_honee_style_setup_links_against_the_library(tmp_path, hb):
    if not os.path.exists(hb.LIB_PATH):
        hb.build()
    src = tmp_path / "setup.c"
    src.write_text(textwrap.dedent(r'''
        #include <ceed.h>
        #include <stdio.h>
        /* the calls of src/setuplibceed.c:209-269 and src/setupts.c:91-109, with error handling as HONEE does it */
        int main(int argc, char **argv) {
          Ceed ceed; CeedQFunction qf; CeedOperator op, comp; CeedQFunctionContext ctx; CeedContextFieldLabel lab;
          const char *msg;
          if (CeedInit("/gpu/b200", &ceed)) { CeedGetErrorMessage(NULL, &msg); printf("init: %s\n", msg); return 0; }
          CeedSetErrorHandler(ceed, CeedErrorStore);
          CeedQFunctionCreateInterior(ceed, 1, NULL, "newtonian.h:IFunction_Newtonian_Conserv", &qf);
          CeedQFunctionAddInput(qf, "q", 5, CEED_EVAL_INTERP);
          CeedOperatorCreate(ceed, qf, NULL, NULL, &op);
          CeedOperatorCreateComposite(ceed, &comp);
          CeedOperatorCompositeAddSub(comp, op);
          CeedQFunctionContextCreate(ceed, &ctx);
          CeedOperatorGetContextFieldLabel(comp, "timestep size", &lab);
          CeedQFunctionContextDestroy(&ctx); CeedOperatorDestroy(&op); CeedOperatorDestroy(&comp); CeedQFunctionDestroy(&qf);
          return CeedDestroy(&ceed);
        }'''))
    exe = tmp_path / "setup"
    libdir = os.path.dirname(hb.LIB_PATH)
    r = subprocess.run(["gcc", "-std=gnu99", f"-I{INC}", str(src), "-o", str(exe), f"-L{libdir}", "-lceed_b200", f"-Wl,-rpath,{libdir}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stdout + run.stderr
