"""The C ABI from C: a C99 program that includes include/gwfa.h (strict C, -Wall -Werror
-pedantic) and links libgwfa_b200.so, as a C caller of the reference's interface would, runs the
entry points that need no GPU: GFA load and dump, read-set load, the host CSR of gwf_ed_index,
and the error codes of calls that need a device or get bad arguments."""
import os
import shutil
import subprocess

import pytest

from conftest import GOLD, PKG_DIR

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "gwfa.h"

int main(int argc, char **argv)
{
	gwf_graph_t *g;
	gwf_reads_t *r;
	int64_t n;
	char *buf;
	int32_t d = 0, st = 0, eo = 0, pn = 0;
	uint32_t v;
	if (argc < 3) return 1;
	g = gwf_gfa_load(argv[1], NULL);
	if (!g) return 2;
	n = gwf_graph_dump(g, NULL, 0);
	buf = (char *)malloc((size_t)n + 1);
	if (gwf_graph_dump(g, buf, n + 1) != n) return 3;
	fwrite(buf, 1, (size_t)n, stdout);
	free(buf);
	r = gwf_reads_load(argv[2]);
	if (!r) return 4;
	fprintf(stderr, "reads %d bases %lld first %d\n", r->n, (long long)r->n_bases, r->n ? r->lens[0] : -1);
	gwf_ed_index(g); /* host CSR always; the device copy fails without a GPU */
	for (v = 0; v < g->n_vtx; ++v)
		if (g->aux[v] >> 32 > g->n_arc) return 5;
	fprintf(stderr, "gwf_ed %d\n", gwf_ed(NULL, g, r->lens[0], r->seqs + r->offs[0], 0, -1, 0, 0));
	fprintf(stderr, "traceback %d\n", gwf_ed(NULL, g, r->lens[0], r->seqs + r->offs[0], 0, -1, 0, 1));
	fprintf(stderr, "path %d\n", gwf_ed_batch_path(g, -1, r->seqs, r->offs, r->lens, &st, -1, 0, 1, &d, &st, &eo,
	                                               &pn, NULL, NULL));
	gwf_reads_free(r);
	gwf_graph_free(g);
	return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_program_uses_the_abi(G, tmp_path):
    G.lib()
    src = tmp_path / "caller.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "caller"
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I" + os.path.join(ROOT, "include"),
                         "-o", str(exe), str(src), "-L" + PKG_DIR, "-lgwfa_b200", "-Wl,-rpath," + PKG_DIR],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe), os.path.join(GOLD, "graph_1000.gfa"), os.path.join(GOLD, "reads_200.fa")],
                         capture_output=True, timeout=120)
    assert run.returncode == 0, run.stderr
    assert run.stdout == open(os.path.join(GOLD, "graph_1000.ref_dump.txt"), "rb").read()
    err = run.stderr.decode()
    assert "reads 200 " in err
    codes = {k: int(v) for k, v in (ln.split() for ln in err.splitlines() if ln.split()[0] in ("gwf_ed", "traceback", "path"))}
    assert codes["traceback"] == G.GWF_E_UNSUPPORTED and codes["path"] == G.GWF_E_BAD_INPUT
    # no device here: the index stays host-only and gwf_ed reports it; with a GPU, a distance
    assert codes["gwf_ed"] in (G.GWF_E_NOT_INDEXED, G.GWF_E_CUDA) or codes["gwf_ed"] >= -1
