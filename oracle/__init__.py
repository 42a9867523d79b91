"""CPU oracle for the llama_b200 engine - test infrastructure only."""
