"""Single-rank stand-in for mpi4py, used only to run the reference PyFlow in this
container when generating golden fixtures.  Semantics follow what
src/library/parallel.py needs: a periodic Cartesian communicator whose Shift
returns the rank itself, Sendrecv that copies the send buffer into the receive
buffer, and Allreduce that copies.  The rank id can be faked through the
PF_FAKE_RANK environment variable (rank 1 skips the reference's rank-0-only
file output)."""
