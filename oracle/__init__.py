"""Host oracle (test infrastructure only): see oracle/fastfft_oracle.py."""
