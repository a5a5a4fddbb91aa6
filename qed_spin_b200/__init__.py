"""qed_spin_b200: the symmetry-sector matvec and the Lanczos / FTLM / continued-fraction recurrences of
QED_Spin's exact diagonalization engine, rebuilt for one NVIDIA B200 (sm_100a) behind a C-ABI."""
__version__ = "0.1.0"
